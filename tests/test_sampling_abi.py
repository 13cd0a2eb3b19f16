"""Host-side checks that need no GPU: the ABI surface and the sampler."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def test_library_exports_every_declared_symbol(t2b):
    header = open(os.path.join(ROOT, "include", "t2b.h")).read()
    declared = set(re.findall(r"\b(t2b_[a-z0-9_]+)\s*\(", header))
    assert declared == set(t2b.ABI_SYMBOLS)
    for name in declared:
        assert hasattr(t2b.lib, name), name
    assert "sm_100a" in t2b.version()


def test_context_creation_without_gpu_fails_cleanly(t2b):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(t2b.T2BError):
        t2b.EStep(0)


@pytest.mark.parametrize("order,npsi,ndir", [(2, 48, 192), (3, 48, 768)])
def test_sampling_counts(t2b, order, npsi, ndir):
    s = t2b.sampling(3, order, 7.5, 1, 3, 1, 2.0)
    assert (s["n_dir"], s["n_psi"], s["nover_rot"], s["nover_trans"]) == (ndir, npsi, 8, 4)
    assert s["n_trans"] == 29
    assert t2b.sampling(3, order, 7.5, 0, 5, 1, 1.3)["n_trans"] == 81
    assert t2b.sampling(3, order, 7.5, 0, 4, 1, 0.85)["n_trans"] == 49


def test_sampling_matches_oracle_healpix(t2b, oracle, synth):
    s = t2b.sampling(3, 2, 7.5, 1, 3, 1, 2.0)
    ang = s["angles"]
    for o in range(0, ang.shape[0], 48):
        z, phi = oracle.healpix_pix2zphi(2, o // 48)
        rot = phi * 180 / np.pi
        tilt = np.arccos(z) * 180. / np.pi
        rot = rot - 360 if rot > 180 else rot
        assert ang[o, 0] == pytest.approx(rot, abs=1e-12)
        assert ang[o, 1] == pytest.approx(tilt, abs=1e-12)
    A = synth.euler_matrix(ang[:, 0], ang[:, 1], ang[:, 2]).reshape(-1, 9)
    assert np.max(np.abs(A - s["eul_coarse"])) < 1e-14
    # fine orientations: the 4 HEALPix children of each direction, 2 psi each,
    # all within one coarse pixel radius of the parent direction
    Ef = s["eul_fine"].reshape(-1, 8, 3, 3)
    Ec = s["eul_coarse"].reshape(-1, 3, 3)
    dots = np.einsum("ok,ork->or", Ec[:, 2, :], Ef[:, :, 2, :])
    assert np.all(dots > np.cos(np.radians(20)))
    # oversampled psi straddle the coarse one by +-psi_step/4
    t = s["trans_px_fine"].reshape(-1, 4, 2) - s["trans_px"][:, None, :]
    assert np.allclose(np.abs(t), 0.25)


def test_sampling_2d(t2b):
    s = t2b.sampling(2, 0, 6.0, 1, 5, 1, 1.0)
    assert (s["n_dir"], s["n_psi"], s["nover_rot"], s["n_trans"]) == (1, 60, 2, 81)
    psi = np.degrees(np.arctan2(s["eul_fine"][:, 1], s["eul_fine"][:, 0]))
    assert np.allclose(np.sort(np.mod(psi, 360))[:4], [1.5, 4.5, 7.5, 10.5])


def test_cpp_adapter_compiles_and_links(tmp_path):
    """The C++ classes a maintainer includes (t2b_adapter.hpp) compile against the
    C ABI and link with libt2b.so (no GPU call is made)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "use_adapter.cpp"
    src.write_text(
        '#include "t2b_adapter.hpp"\n'
        "int main(int argc, char**) {\n"
        "  if (argc > 5) {  // never taken: only the symbols are needed\n"
        "    t2b::MlDeviceBundle b(0);\n"
        "    t2b::MlOptimiserCuda opt(b);\n"
        "    t2b::ProposalNetwork net(b);\n"
        "    net.enable();\n"
        "    t2b::AccBackprojector bp(b, 0);\n"
        "  }\n"
        "  return 0;\n"
        "}\n")
    lib_dir = os.path.join(ROOT, "t2-relion_b200")
    out = tmp_path / "use_adapter"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-L", lib_dir, "-lt2b",
                        "-Wl,--unresolved-symbols=ignore-in-shared-libs", "-o", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("order,psi,rng,angpix", [(1, 15.0, 3, 2.0), (3, 7.5, 5, 1.3)])
def test_sampling_matches_oracle_restatement(t2b, order, psi, rng, angpix):
    """The library's sampler against the oracle's numpy restatement of HealpixSampling (the lists
    the reference arm of the benchmark uses): identical translations, matrices within 1e-15."""
    import sampling_oracle as so
    a = t2b.sampling(3, order, psi, 1, rng, 1, angpix)
    b = so.sampling(order, psi, 1, rng, 1, angpix)
    for k in ("n_dir", "n_psi", "n_trans", "nover_rot", "nover_trans"):
        assert a[k] == b[k], k
    for k in ("trans_px", "trans_px_fine", "trans_prior"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("eul_coarse", "eul_fine"):
        assert np.max(np.abs(a[k] - b[k])) <= 1e-15, k


def test_sampling_2d_matches_oracle_restatement(t2b):
    import sampling_oracle as so
    a = t2b.sampling(2, 0, 6.0, 1, 5, 1, 2.0)
    b = so.sampling2d(6.0, 1, 5, 1, 2.0)
    for k in ("n_dir", "n_psi", "n_trans", "nover_rot", "nover_trans"):
        assert a[k] == b[k], k
    for k in ("trans_px", "trans_px_fine", "trans_prior"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("eul_coarse", "eul_fine"):
        assert np.max(np.abs(a[k] - b[k])) <= 1e-15, k
