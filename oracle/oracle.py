"""ctypes front end of the FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The shipped library never uses it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_HP = os.path.join(HERE, "_ref", "libhp_ref.so")


def build(ref=True):
    """Compile the oracle (and, when the reference tree is present, oracle/_ref)."""
    targets = ["liboracle.so"]
    if ref and os.path.isdir(os.environ.get("REF", "/root/reference")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _lib():
    if not os.path.exists(LIB):
        build(ref=False)
    return ctypes.CDLL(LIB)


L = _lib()
_p = ctypes.c_void_p


class Setup(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "ori_size", "s", "ref_dim", "nr_classes", "n_dir", "n_psi", "n_trans", "nover_rot",
        "nover_trans", "adaptive_oversampling", "maximum_significants")] + [
        ("maps", _p)] + [(n, ctypes.c_int) for n in (
            "mxdim", "mydim", "mzdim", "minity", "minitz", "mr_max", "mpad")] + [
        (n, _p) for n in ("eul_coarse", "eul_fine", "trans_px", "trans_px_fine", "trans_prior",
                          "pdf_direction", "pdf_class")] + [
        ("sigma2_offset", ctypes.c_double), ("pixel_size", ctypes.c_double),
        ("adaptive_fraction", ctypes.c_double), ("bp_data", _p), ("bp_weight", _p)] + [
        (n, ctypes.c_int) for n in ("bxdim", "bydim", "bzdim", "binity", "binitz", "br_max", "bpad")] + [
        ("data_vs_prior", _p)]


class Particle(ctypes.Structure):
    _fields_ = [("fimg", _p), ("fimg_nomask", _p), ("ctf", _p), ("minvsigma2", _p), ("mresol", _p),
                ("minvsigma2_dc", ctypes.c_double), ("highres_xi2", ctypes.c_double),
                ("old_offset", ctypes.c_double * 2), ("prior", ctypes.c_double * 2),
                ("scale", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("min_diff2", ctypes.c_double), ("sum_weight", ctypes.c_double),
                ("sig_weight", ctypes.c_double), ("coarse_min_diff2", ctypes.c_double),
                ("coarse_sum_weight", ctypes.c_double), ("coarse_sig_weight", ctypes.c_double),
                ("nr_sign", ctypes.c_longlong), ("n_coarse_sig", ctypes.c_longlong),
                ("pmax", ctypes.c_double), ("pose", ctypes.c_int * 5), ("wsum_norm", ctypes.c_double),
                ("sumw", ctypes.c_double), ("wsum_sigma2_offset", ctypes.c_double),
                ("wsum_scale_xa", ctypes.c_double), ("wsum_scale_aa", ctypes.c_double)]


L.orc_ctf_value.restype = ctypes.c_double
L.orc_ctf_value.argtypes = [_p, ctypes.c_double, ctypes.c_double]
L.orc_ctf_image.argtypes = [_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _p]
L.orc_project.argtypes = [ctypes.POINTER(Setup), ctypes.c_int, _p, _p]
L.orc_coarse_diff2.restype = ctypes.c_double
L.orc_coarse_diff2.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), _p]
L.orc_weights.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), ctypes.c_int, _p, _p,
                          ctypes.c_longlong, ctypes.c_double, _p, _p, _p, _p]
L.orc_fine_diff2.restype = ctypes.c_longlong
L.orc_fine_diff2.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), _p, _p, _p, _p]
L.orc_estep.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), ctypes.c_int,
                        ctypes.POINTER(Result), _p, _p, _p, ctypes.c_int]
L.orc_wsum_bp.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), _p, ctypes.c_longlong, _p,
                          ctypes.c_double, ctypes.c_double, ctypes.POINTER(Result), _p, _p, _p]
L.orc_diff2_literal.restype = ctypes.c_double
L.orc_diff2_literal.argtypes = [ctypes.POINTER(Setup), ctypes.POINTER(Particle), ctypes.c_int, _p,
                                ctypes.c_double, ctypes.c_double]
L.orc_reconstruct_divide.argtypes = [_p, _p] + [ctypes.c_int] * 7 + [_p]
L.orc_healpix_nest_pix2zphi.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_p)


def ctf_value(params, X, Y):
    p = np.ascontiguousarray(params, np.float64)
    return L.orc_ctf_value(_ptr(p), X, Y)


def ctf_image(params, ori_size, angpix, s):
    p = np.ascontiguousarray(params, np.float64)
    out = np.zeros(s * (s // 2 + 1), np.float32)
    L.orc_ctf_image(_ptr(p), ori_size, angpix, s, _ptr(out))
    return out


def healpix_pix2zphi(order, pix):
    z, phi = ctypes.c_double(), ctypes.c_double()
    L.orc_healpix_nest_pix2zphi(order, pix, ctypes.byref(z), ctypes.byref(phi))
    return z.value, phi.value


class Problem:
    """Holds the numpy arrays an OrcSetup points to (keeps them alive)."""

    def __init__(self, *, ori_size, s, ref_dim, maps, r_max, pad, samp, pdf_direction, pdf_class,
                 sigma2_offset, pixel_size, adaptive_fraction, ovs, bp_pad_size, bp_r_max, maximum_significants=-1,
                 data_vs_prior=None):
        self.maps = np.ascontiguousarray(np.stack(maps), np.complex64)
        self.eul_coarse = np.ascontiguousarray(samp["eul_coarse"], np.float64)
        self.eul_fine = np.ascontiguousarray(samp["eul_fine"], np.float64)
        self.trans_px = np.ascontiguousarray(samp["trans_px"], np.float64)
        self.trans_px_fine = np.ascontiguousarray(samp["trans_px_fine"], np.float64)
        self.trans_prior = np.ascontiguousarray(samp["trans_prior"], np.float64)
        self.pdf_direction = np.ascontiguousarray(pdf_direction, np.float64)
        self.pdf_class = np.ascontiguousarray(pdf_class, np.float64)
        K = len(maps)
        m0 = maps[0]
        if ref_dim == 3:
            mz, my, mx = m0.shape
            bz = bp_pad_size
            gshape = (K, bz, bp_pad_size, bp_pad_size // 2 + 1)
        else:
            my, mx = m0.shape
            mz = 1
            bz = 1
            gshape = (K, bp_pad_size, bp_pad_size // 2 + 1)
        self.gshape = gshape
        self.bp_data = np.zeros(gshape + (2,), np.float64)
        self.bp_weight = np.zeros(gshape, np.float64)
        S = Setup()
        S.ori_size, S.s, S.ref_dim, S.nr_classes = ori_size, s, ref_dim, K
        S.n_dir, S.n_psi, S.n_trans = samp["n_dir"], samp["n_psi"], samp["n_trans"]
        S.nover_rot = samp["nover_rot"] if ovs else 1
        S.nover_trans = samp["nover_trans"] if ovs else 1
        S.adaptive_oversampling, S.maximum_significants = ovs, maximum_significants
        S.maps = _ptr(self.maps)
        S.mxdim, S.mydim, S.mzdim = mx, my, mz
        S.minity, S.minitz = -(my // 2), (-(mz // 2) if ref_dim == 3 else 0)
        S.mr_max, S.mpad = r_max, pad
        for k in ("eul_coarse", "eul_fine", "trans_px", "trans_px_fine", "trans_prior",
                  "pdf_direction", "pdf_class"):
            setattr(S, k, _ptr(getattr(self, k)))
        S.sigma2_offset, S.pixel_size, S.adaptive_fraction = sigma2_offset, pixel_size, adaptive_fraction
        S.bp_data, S.bp_weight = _ptr(self.bp_data), _ptr(self.bp_weight)
        S.bxdim, S.bydim, S.bzdim = bp_pad_size // 2 + 1, bp_pad_size, bz
        S.binity, S.binitz = -(bp_pad_size // 2), (-(bp_pad_size // 2) if ref_dim == 3 else 0)
        S.br_max, S.bpad = bp_r_max, pad
        self.data_vs_prior = None if data_vs_prior is None else np.ascontiguousarray(data_vs_prior, np.float64)
        S.data_vs_prior = _ptr(self.data_vs_prior)
        self.S = S
        self.half = ori_size // 2 + 1
        self.K, self.n_dir = K, samp["n_dir"]
        self.O = samp["n_dir"] * samp["n_psi"]
        self.T = samp["n_trans"]
        self.RV = S.nover_rot * S.nover_trans
        self.mresol = None

    def particles(self, fimg, ctf, minv, scalars, mresol, fimg_nomask=None):
        self._pin = [np.ascontiguousarray(fimg, np.complex64), np.ascontiguousarray(ctf, np.float32),
                     np.ascontiguousarray(minv, np.float32), np.ascontiguousarray(mresol, np.int32),
                     None if fimg_nomask is None else np.ascontiguousarray(fimg_nomask, np.complex64)]
        f, c, m, mr, fn = self._pin
        n = f.shape[0]
        arr = (Particle * n)()
        for b in range(n):
            pt = arr[b]
            pt.fimg = f[b].ctypes.data
            pt.fimg_nomask = (fn[b] if fn is not None else f[b]).ctypes.data
            pt.ctf = c[b].ctypes.data
            pt.minvsigma2 = m[b].ctypes.data
            pt.mresol = mr.ctypes.data
            sc = scalars[b]
            pt.minvsigma2_dc, pt.highres_xi2 = sc[0], sc[1]
            pt.old_offset[0], pt.old_offset[1] = sc[2], sc[3]
            pt.prior[0], pt.prior[1] = sc[4], sc[5]
            pt.scale = sc[6]
        return arr

    def project(self, iclass, A):
        s = self.S.s
        out = np.zeros(2 * s * (s // 2 + 1))
        a = np.ascontiguousarray(A, np.float64).reshape(9)
        L.orc_project(ctypes.byref(self.S), iclass, _ptr(a), _ptr(out))
        return out[0::2] + 1j * out[1::2]

    def coarse_diff2(self, parts, b):
        out = np.zeros(self.K * self.O * self.T)
        mn = L.orc_coarse_diff2(ctypes.byref(self.S), ctypes.byref(parts[b]), _ptr(out))
        return out, mn

    def weights(self, parts, b, ipass, diff2, ihidden, min_diff2):
        d = np.ascontiguousarray(diff2, np.float64)
        ih = np.ascontiguousarray(ihidden, np.int64)
        w = np.zeros(d.size)
        sw, sg = ctypes.c_double(), ctypes.c_double()
        ns = ctypes.c_longlong()
        rc = L.orc_weights(ctypes.byref(self.S), ctypes.byref(parts[b]), ipass, _ptr(d), _ptr(ih), d.size,
                           min_diff2, _ptr(w), ctypes.byref(sw), ctypes.byref(sg), ctypes.byref(ns))
        return rc, w, sw.value, sg.value, ns.value

    def fine_diff2(self, parts, b, mask):
        m = np.ascontiguousarray(mask, np.uint8)
        cap = int(m.sum())
        pairs = np.zeros(max(cap, 1), np.int64)
        out = np.zeros(max(cap, 1) * self.RV)
        mn = ctypes.c_double()
        np_ = L.orc_fine_diff2(ctypes.byref(self.S), ctypes.byref(parts[b]), _ptr(m), _ptr(pairs), _ptr(out),
                               ctypes.byref(mn))
        return pairs[:np_], out[:np_ * self.RV].reshape(np_, self.RV), mn.value

    def estep(self, parts, nthreads=0):
        n = len(parts)
        res = (Result * n)()
        sig = np.zeros((n, self.half))
        pc = np.zeros((n, self.K))
        pd = np.zeros((n, self.K * self.n_dir))
        nthreads = nthreads or os.cpu_count() or 1
        fails = L.orc_estep(ctypes.byref(self.S), parts, n, res, _ptr(sig), _ptr(pc), _ptr(pd), nthreads)
        out = {k: np.array([getattr(r, k) for r in res]) for k, _ in Result._fields_ if k != "pose"}
        out["pose"] = np.array([list(r.pose) for r in res])
        out.update(wsum_sigma2=sig, wsum_pdf_class=pc, wsum_pdf_dir=pd, fails=fails)
        return out

    def wsum_bp(self, parts, b, pairs, wf, fsum, fsig):
        """Weighted sums + backprojection of particle b on given final weights (the oracle's
        stage on the same input as the device's); grids accumulate into this Problem's."""
        pr = np.ascontiguousarray(pairs, np.int64)
        w = np.ascontiguousarray(wf, np.float64)
        res = Result()
        sig = np.zeros(self.half)
        pc = np.zeros(self.K)
        pd = np.zeros(self.K * self.n_dir)
        L.orc_wsum_bp(ctypes.byref(self.S), ctypes.byref(parts[b]), _ptr(pr), pr.size, _ptr(w), fsum, fsig,
                      ctypes.byref(res), _ptr(sig), _ptr(pc), _ptr(pd))
        out = {k: getattr(res, k) for k, _ in Result._fields_ if k != "pose"}
        out["pose"] = np.array(list(res.pose))
        out.update(wsum_sigma2=sig, wsum_pdf_class=pc, wsum_pdf_dir=pd)
        return out

    def diff2_literal(self, parts, b, iclass, A, shift):
        a = np.ascontiguousarray(A, np.float64).reshape(9)
        return L.orc_diff2_literal(ctypes.byref(self.S), ctypes.byref(parts[b]), iclass, _ptr(a),
                                   float(shift[0]), float(shift[1]))

    def clear_grids(self):
        self.bp_data[...] = 0
        self.bp_weight[...] = 0

    def grids(self):
        return self.bp_data[..., 0] + 1j * self.bp_data[..., 1], self.bp_weight


def reconstruct_divide(data, weight, r_max, pad):
    """data: complex (pad, pad, pad//2+1) centred grid; returns FFTW-ordered Fconv."""
    ps = data.shape[1]
    d = np.ascontiguousarray(np.stack([data.real, data.imag], -1), np.float64)
    w = np.ascontiguousarray(weight, np.float64)
    out = np.zeros((ps, ps, ps // 2 + 1, 2))
    L.orc_reconstruct_divide(_ptr(d), _ptr(w), ps // 2 + 1, ps, ps, -(ps // 2), -(ps // 2), r_max, pad, _ptr(out))
    return out[..., 0] + 1j * out[..., 1]
