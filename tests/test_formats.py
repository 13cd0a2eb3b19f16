"""On-disk formats (CPU): the library's STAR parser against the reference's own
MetaDataTable (compiled from its sources into oracle/_ref/libstar_ref.so), and
the MRC reader / writer against the MRC2014 layout restated with numpy (modes
0, 1, 2, 6, 12, extended headers, byte-swapped files; every half-precision bit
pattern)."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT

PARTICLES_STAR = """
# version 30001

data_optics

loop_
_rlnOpticsGroupName #1
_rlnOpticsGroup #2
_rlnMtfFileName #3
_rlnMicrographOriginalPixelSize #4
_rlnVoltage #5
_rlnSphericalAberration #6
_rlnAmplitudeContrast #7
_rlnImagePixelSize #8
_rlnImageSize #9
_rlnImageDimensionality #10
opticsGroup1            1 mtf_k2_200kV.star     0.885000   200.000000     1.400000     0.100000     1.770000          64            2


# version 30001

data_particles

loop_
_rlnCoordinateX #1
_rlnCoordinateY #2
_rlnAnglePsi #3
_rlnClassNumber #4
_rlnAutopickFigureOfMerit #5
_rlnImageName #6
_rlnMicrographName #7
_rlnOpticsGroup #8
_rlnCtfMaxResolution #9
_rlnCtfFigureOfMerit #10
_rlnDefocusU #11
_rlnDefocusV #12
_rlnDefocusAngle #13
_rlnCtfBfactor #14
_rlnCtfScalefactor #15
_rlnPhaseShift #16
_rlnOriginXAngst #17
_rlnOriginYAngst #18
_rlnAngleRot #19
_rlnAngleTilt #20
_rlnNormCorrection #21
_rlnSomeLabelNobodyKnows #22
  1614.217  1164.436   -999.00000   1   2.004727 000001@Extract/job007/Movies/20170629_00021_frameImage.mrcs MotionCorr/job002/Movies/20170629_00021_frameImage.mrc 1 4.809192 0.131159 10863.857422 10575.166016 77.997299 0.000000 1.000000 0.000000 -3.540000 1.770000 -12.5 90.0 1.0 xyz
  1200.000  1100.000   -999.00000   1   1.5e-1 000002@Extract/job007/Movies/20170629_00021_frameImage.mrcs MotionCorr/job002/Movies/20170629_00021_frameImage.mrc 1 4.809192 0.131159 10863.857422 10575.166016 77.997299 0.000000 1.000000 0.000000 0.885000 -0.885 170.25 35.5 0.97 abc
  300.5  -20   12.5   2   -2.5E+2 '000003@Extract/job007/Movies/a b.mrcs' "MotionCorr/job002/Movies/x.mrc" 1 3.5 0.2 20000.0 19500.25 -45.0 12.0 0.9 10.0 0 0 0 0 1 q

data_model_general

_rlnReferenceDimensionality                        3
_rlnDataDimensionality                             2
_rlnOriginalImageSize                            64
_rlnCurrentResolution                            12.345600
_rlnPixelSize                                    1.770000
_rlnTau2FudgeFactor                              1.000000
_rlnReferenceDimensionality2                      unknown
"""


def _ref_star():
    path = os.path.join(ROOT, "oracle", "_ref", "libstar_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference STAR reader not built (needs the reference tree)")
    L = ctypes.CDLL(path)
    L.ref_star_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    L.ref_star_get_double.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.POINTER(ctypes.c_double)]
    L.ref_star_get_string.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_char_p, ctypes.c_int]
    return L


@pytest.mark.parametrize("block", ["optics", "particles", "model_general"])
def test_star_matches_reference_reader(t2b, tmp_path, block):
    ref = _ref_star()
    fn = tmp_path / "particles.star"
    fn.write_text(PARTICLES_STAR)
    tab = t2b.StarTable(str(fn), block)
    n = ref.ref_star_read(str(fn).encode(), block.encode())
    assert n == tab.rows and n >= 1
    checked = 0
    for lab in tab.labels:
        v = ctypes.c_double()
        if ref.ref_star_get_double(lab.encode(), 0, ctypes.byref(v)) == -2:
            continue              # a label the reference does not know (kept as text by both)
        try:
            ours = tab.column(lab)
        except t2b.T2BError:      # a text column: compare the text
            buf = ctypes.create_string_buffer(1024)
            for r in range(n):
                assert ref.ref_star_get_string(lab.encode(), r, buf, 1024) == 0
                assert tab.value(lab, r) == buf.value.decode(), (lab, r)
            checked += 1
            continue
        for r in range(n):
            assert ref.ref_star_get_double(lab.encode(), r, ctypes.byref(v)) == 0
            assert ours[r] == v.value, (lab, r, ours[r], v.value)
        checked += 1
    assert checked >= min(len(tab.labels), 6)


def test_star_quoted_and_unknown_values(t2b, tmp_path):
    fn = tmp_path / "p.star"
    fn.write_text(PARTICLES_STAR)
    tab = t2b.StarTable(str(fn), "particles")
    assert tab.rows == 3 and len(tab.labels) == 22
    assert tab.value("rlnImageName", 2) == "000003@Extract/job007/Movies/a b.mrcs"
    assert tab.value("rlnSomeLabelNobodyKnows", 1) == "abc"
    assert np.allclose(tab.column("rlnAutopickFigureOfMerit"), [2.004727, 0.15, -250.0])
    first = t2b.StarTable(str(fn))
    assert first.labels[0] == "rlnOpticsGroupName" and first.rows == 1
    with pytest.raises(t2b.T2BError):
        t2b.StarTable(str(fn), "nonexistent")


def test_star_comment_line_inside_a_loop_is_skipped(t2b, tmp_path):
    """(The reference's reader stops with an error on such a line; this parser skips it.)"""
    text = PARTICLES_STAR.replace("  300.5", "# a comment line inside the loop\n  300.5")
    fn = tmp_path / "c.star"
    fn.write_text(text)
    tab = t2b.StarTable(str(fn), "particles")
    assert tab.rows == 3 and tab.column("rlnCoordinateX")[2] == 300.5


def test_star_write_read_roundtrip(t2b, tmp_path):
    ref = _ref_star()
    rng = np.random.default_rng(0)
    cols = {"rlnAngleRot": rng.uniform(-180, 180, 50), "rlnAngleTilt": rng.uniform(0, 180, 50),
            "rlnOriginXAngst": rng.normal(0, 3, 50), "rlnClassNumber": rng.integers(1, 5, 50).astype(float)}
    fn = tmp_path / "out.star"
    t2b.write_star(str(fn), "particles", cols)
    t2b.write_star(str(fn), "extra", {"rlnPixelSize": [1.25]}, append=True)
    tab = t2b.StarTable(str(fn), "particles")
    for k, v in cols.items():
        assert np.array_equal(tab.column(k), v)
    assert t2b.StarTable(str(fn), "extra").column("rlnPixelSize")[0] == 1.25
    assert ref.ref_star_read(str(fn).encode(), b"particles") == 50
    x = ctypes.c_double()
    for r in (0, 17, 49):
        ref.ref_star_get_double(b"rlnAngleRot", r, ctypes.byref(x))
        assert x.value == cols["rlnAngleRot"][r]


# ---------------------------------------------------------------- MRC
def _mrc_header(nx, ny, nz, mode, apix, nsymbt=0):
    """MRC2014 header (1024 bytes): words 1-10 int32, 11-16 float (cell), 17-19 int32,
    20-22 float, 23-24 int32, 50-52 origin, 53 'MAP ', 54 machine stamp, 55 rms, 56 nlabl."""
    h = np.zeros(256, np.int32)
    h[0:4] = nx, ny, nz, mode
    h[7:10] = nx, ny, nz
    f = h.view(np.float32)
    f[10:13] = apix * nx, apix * ny, apix * nz
    f[13:16] = 90.0
    h[16:19] = 1, 2, 3
    h[23] = nsymbt
    h[52] = np.frombuffer(b"MAP ", np.int32)[0]
    h[53] = np.frombuffer(bytes([0x44, 0x41, 0, 0]), np.int32)[0]
    return h


def _write_raw(path, header, data, nsymbt=0, swap=False):
    with open(path, "wb") as fo:
        hh = header.copy()
        if swap:
            hh[:56] = hh[:56].byteswap()
        fo.write(hh.tobytes())
        fo.write(b"\x01" * nsymbt)
        fo.write((data.byteswap() if swap else data).tobytes())


@pytest.mark.parametrize("mode,dtype", [(0, np.int8), (1, np.int16), (2, np.float32), (6, np.uint16),
                                        (12, np.float16)])
@pytest.mark.parametrize("swap", [False, True], ids=["little", "swapped"])
def test_mrc_modes(t2b, tmp_path, mode, dtype, swap):
    rng = np.random.default_rng(mode)
    nx, ny, nz = 24, 20, 5
    if dtype == np.float16 or dtype == np.float32:
        data = rng.normal(0, 3, (nz, ny, nx)).astype(dtype)
    else:
        info = np.iinfo(dtype)
        data = rng.integers(info.min, info.max, (nz, ny, nx), endpoint=True).astype(dtype)
    fn = str(tmp_path / f"m{mode}.mrcs")
    _write_raw(fn, _mrc_header(nx, ny, nz, mode, 1.77, nsymbt=96), data, nsymbt=96, swap=swap)
    assert t2b.mrc_info(fn)[:4] == (nx, ny, nz, mode)
    assert t2b.mrc_info(fn)[4] == pytest.approx(1.77, rel=1e-6)
    got = t2b.read_mrc(fn, 1, 3)
    assert np.array_equal(got, data[1:4].astype(np.float32))


def test_half_precision_every_bit_pattern(t2b, tmp_path):
    bits = np.arange(65536, dtype=np.uint16).reshape(256, 256, 1)[:, :, 0].reshape(1, 256, 256)
    fn = str(tmp_path / "h.mrc")
    _write_raw(fn, _mrc_header(256, 256, 1, 12, 1.0), bits)
    got = t2b.read_mrc(fn)
    want = bits.view(np.float16).astype(np.float32)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    assert np.array_equal(got[~nan], want[~nan])
    assert np.array_equal(np.signbit(got[~nan]), np.signbit(want[~nan]))


def test_mrc_write_matches_layout(t2b, tmp_path):
    rng = np.random.default_rng(3)
    vol = rng.normal(0, 1, (7, 16, 12)).astype(np.float32)
    fn = str(tmp_path / "w.mrc")
    t2b.write_mrc(fn, vol, 1.3)
    raw = np.fromfile(fn, np.uint8)
    h = raw[:1024].view(np.int32)
    assert tuple(h[0:4]) == (12, 16, 7, 2) and tuple(h[7:10]) == (12, 16, 7)
    assert raw[:1024].view(np.float32)[10] == pytest.approx(1.3 * 12)
    assert bytes(raw[208:212]) == b"MAP "
    assert np.array_equal(raw[1024:].view(np.float32).reshape(7, 16, 12), vol)
    assert np.array_equal(t2b.read_mrc(fn), vol)


def test_prep_parameters_from_star(t2b, tmp_path):
    fn = tmp_path / "p.star"
    fn.write_text(PARTICLES_STAR)
    tab = t2b.StarTable(str(fn), "particles")
    par = t2b.prep_params_from_star(tab, 1.77)
    assert par.shape == (3, t2b.PREP_NPARAM)
    assert np.allclose(par[:, 0], np.array([-3.54, 0.885, 0.0]) / 1.77)
    assert np.allclose(par[:, 1], np.array([1.77, -0.885, 0.0]) / 1.77)
    assert np.all(par[:, 2:4] == 999.0)
    assert np.allclose(par[:, 4], [1.0, 0.97, 1.0])
    assert np.allclose(par[:, 5:8], tab.column("rlnDefocusU")[:, None] * [1, 0, 0] +
                       tab.column("rlnDefocusV")[:, None] * [0, 1, 0] + tab.column("rlnDefocusAngle")[:, None] * [0, 0, 1])
    assert np.allclose(par[:, 8], [0.0, 0.0, 12.0]) and np.allclose(par[:, 10], [0.0, 0.0, 10.0])
