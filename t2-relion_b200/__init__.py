"""Host-side mirror of the RELION E-step accelerator interface over libt2b.so.

The reference drives its GPU E-step through C++ classes: AccProjector
(src/acc/acc_projector.h:69-78), AccBackprojector (src/acc/acc_backprojector.h:
51-79), MlDeviceBundle and MlOptimiserCuda (src/acc/cuda/cuda_ml_optimiser.h:
17-186).  This module exposes the same surface in Python on top of the C ABI in
include/t2b.h; include/t2b_adapter.hpp does the same for C++ callers.

Every call goes to the CUDA library.  There is no CPU fallback: importing this
package fails loudly when libt2b.so is missing, and every non-zero status of
the C ABI raises T2BError with the library's message.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libt2b.so")

T2B_OK = 0
T2B_ERR_ARG = 1
T2B_ERR_CUDA = 2
T2B_ERR_NOSIGNIF = 3
T2B_ERR_STATE = 4
T2B_ERR_NOMEM = 5
T2B_ERR_TIMEOUT = 6
T2B_ERR_UNSUPPORTED = 7
DIFF2_PLAIN_FP32 = 0
DIFF2_SPLIT_BF16 = 1

# every symbol include/t2b.h declares
ABI_SYMBOLS = (
    "t2b_create", "t2b_destroy", "t2b_last_error", "t2b_version",
    "t2b_projector_set", "t2b_backprojector_init", "t2b_backprojector_clear",
    "t2b_backprojector_get", "t2b_backprojector_device_ptrs", "t2b_configure",
    "t2b_estep_batch_host", "t2b_estep_batch_device", "t2b_estep_submit_host", "t2b_estep_wait",
    "t2b_reconstruct_divide",
    "t2b_project", "t2b_debug_coarse_diff2", "t2b_debug_fine", "t2b_debug_weights", "t2b_debug_selection",
    "t2b_debug_proposals", "t2b_last_stage_ms",
    "t2b_sampling", "t2b_reconstruct_divide_noalloc", "t2b_last_launch_count",
    "t2b_proposal_train", "t2b_proposal_enable", "t2b_proposal_params", "t2b_proposal_features",
    "t2b_proposal_logits", "t2b_proposal_grad", "t2b_stage_timing",
    "t2b_prep_configure", "t2b_prep_batch_host", "t2b_prep_batch_device", "t2b_autotune", "t2b_tune_set",
    "t2b_reconstruct", "t2b_fsc_halves", "t2b_update_ssnr", "t2b_backprojector_enforce_hermitian",
    "t2b_point_group", "t2b_backprojector_apply_symmetry", "t2b_backprojector_apply_helical",
    "t2b_mrc_info", "t2b_mrc_read", "t2b_mrc_write", "t2b_star_open", "t2b_star_shape", "t2b_star_label",
    "t2b_star_column", "t2b_star_value", "t2b_star_close", "t2b_star_write",
)


class T2BError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"t2b error {code}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with t2-relion_b200/build.py "
                          "(__graft_entry__.build()); there is no CPU fallback")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_p = ctypes.c_void_p
_d = ctypes.POINTER(ctypes.c_double)


class Config(ctypes.Structure):
    _fields_ = [
        ("ori_size", ctypes.c_int), ("current_size", ctypes.c_int), ("ref_dim", ctypes.c_int),
        ("nr_classes", ctypes.c_int), ("n_dir", ctypes.c_int), ("n_psi", ctypes.c_int),
        ("n_trans", ctypes.c_int), ("adaptive_oversampling", ctypes.c_int),
        ("nover_rot", ctypes.c_int), ("nover_trans", ctypes.c_int),
        ("maximum_significants", ctypes.c_int), ("diff2_mode", ctypes.c_int),
        ("max_batch", ctypes.c_int), ("use_graph", ctypes.c_int),
        ("eul_coarse", _p), ("eul_fine", _p), ("trans_px", _p), ("trans_px_fine", _p),
        ("trans_prior", _p), ("pdf_direction", _p), ("pdf_class", _p), ("mresol", _p),
        ("sigma2_offset", ctypes.c_double), ("pixel_size", ctypes.c_double),
        ("adaptive_fraction", ctypes.c_double), ("fine_capacity", ctypes.c_size_t),
        ("data_vs_prior", _p), ("orientation_chunk", ctypes.c_int), ("_pad2", ctypes.c_int),
    ]


class Batch(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("_pad", ctypes.c_int), ("fimg", _p), ("fimg_nomask", _p),
                ("ctf", _p), ("minvsigma2", _p), ("scalars", _p)]


class Result(ctypes.Structure):
    _fields_ = [(name, _p) for name in (
        "min_diff2", "sum_weight", "sig_weight", "coarse_sum_weight", "coarse_sig_weight",
        "nr_sign", "n_coarse_sig", "pmax", "pose", "wsum_norm", "sumw", "wsum_sigma2_offset",
        "wsum_sigma2", "wsum_pdf_class", "wsum_pdf_dir", "status", "audit_mass", "learned",
        "wsum_scale_xa", "wsum_scale_aa")]


class ProposalTrainConfig(ctypes.Structure):
    _fields_ = [("n_train", ctypes.c_int), ("n_posterior", ctypes.c_int), ("n_val", ctypes.c_int),
                ("epochs", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_float),
                ("topk", ctypes.c_int), ("rescore", ctypes.c_int), ("seed", ctypes.c_ulonglong),
                ("defocus_min", ctypes.c_double), ("defocus_max", ctypes.c_double),
                ("astig_max", ctypes.c_double), ("voltage", ctypes.c_double), ("cs", ctypes.c_double),
                ("q0", ctypes.c_double), ("max_shift", ctypes.c_double), ("sigma_deg", ctypes.c_double),
                ("alpha", ctypes.c_float), ("minvsigma2", _p)]


class ProposalReport(ctypes.Structure):
    _fields_ = [("loss", ctypes.c_double * 64), ("val_mass_init", ctypes.c_double),
                ("val_mass_trained", ctypes.c_double), ("val_mass_min", ctypes.c_double),
                ("val_frac_999", ctypes.c_double), ("val_true_hit", ctypes.c_double),
                ("val_mass_rescored", ctypes.c_double), ("val_mass_min_rescored", ctypes.c_double),
                ("val_frac_999_rescored", ctypes.c_double), ("val_frac_999_candidates", ctypes.c_double),
                ("gen_ms", ctypes.c_double), ("label_ms", ctypes.c_double), ("train_ms", ctypes.c_double),
                ("params", ctypes.c_longlong)]


class PrepConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "image_size", "current_size", "max_batch", "zero_mask", "random_seed", "do_norm_correction",
        "do_ctf_correction", "ctf_premultiplied", "ctf_phase_flipped", "only_flip_phases",
        "intact_ctf_first_peak", "n_sigma2")] + [("sigma2_noise", _p)] + [(n, ctypes.c_double) for n in (
            "pixel_size", "mask_radius", "width_mask_edge", "avg_norm_correction", "sigma2_fudge",
            "remap_noise", "remap_minv", "voltage", "cs", "q0")]


class PrepBatch(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("_pad", ctypes.c_int), ("images", _p), ("params", _p), ("part_id", _p)]


class PrepOut(ctypes.Structure):
    _fields_ = [(n, _p) for n in ("fimg", "fimg_nomask", "ctf", "minvsigma2", "scalars", "power")]


class ReconConfig(ctypes.Structure):
    _fields_ = [("ori_size", ctypes.c_int), ("do_map", ctypes.c_int), ("minres_map", ctypes.c_int),
                ("gridding_iter", ctypes.c_int), ("tau2_fudge", ctypes.c_double), ("tau2", _p),
                ("normalise", ctypes.c_double)]


class SsnrConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("ori_size", "update_tau2_with_fsc", "is_whole_instead_of_half",
                                            "correct_tau2_by_avgctf2")] + [
        ("tau2_fudge", ctypes.c_double), ("fsc", _p), ("avgctf2", _p)]


class TuneReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("diff2_tn", "diff2_group", "fine_ctas_per_sm", "wsum_ctas_per_sm",
                                            "project_pixels", "project_orients")] + [
        ("diff2_ms", ctypes.c_float * 8), ("fine_ms", ctypes.c_float * 4), ("wsum_ms", ctypes.c_float * 4),
        ("project_ms", ctypes.c_float * 9)]


PREP_NPARAM = 12
PREP_DEFAULTS = dict(zero_mask=0, random_seed=0, do_norm_correction=0, do_ctf_correction=1, ctf_premultiplied=0,
                     ctf_phase_flipped=0, only_flip_phases=0, intact_ctf_first_peak=0, avg_norm_correction=1.0,
                     sigma2_fudge=1.0, remap_noise=1.0, remap_minv=1.0, voltage=300.0, cs=2.7, q0=0.1,
                     width_mask_edge=5.0)


def _setup_prototypes():
    i, v, c = ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p
    lib.t2b_create.argtypes = [i, ctypes.POINTER(v)]
    lib.t2b_destroy.argtypes = [v]
    lib.t2b_destroy.restype = None
    lib.t2b_last_error.restype = c
    lib.t2b_version.restype = c
    lib.t2b_projector_set.argtypes = [v, i, i, i, i, i, i, i, i, i, v]
    lib.t2b_backprojector_init.argtypes = [v, i, i, i, i, i, i, i, i, i]
    lib.t2b_backprojector_clear.argtypes = [v, i]
    lib.t2b_backprojector_enforce_hermitian.argtypes = [v, i]
    lib.t2b_point_group.argtypes = [ctypes.c_char_p, v, i, ctypes.POINTER(i)]
    lib.t2b_backprojector_apply_symmetry.argtypes = [v, i, ctypes.c_char_p]
    lib.t2b_backprojector_apply_helical.argtypes = [v, i, i, ctypes.c_double, ctypes.c_double, i]
    lib.t2b_backprojector_get.argtypes = [v, i, v, v, v]
    lib.t2b_backprojector_device_ptrs.argtypes = [v, i, ctypes.POINTER(v), ctypes.POINTER(v)]
    lib.t2b_configure.argtypes = [v, ctypes.POINTER(Config)]
    lib.t2b_estep_batch_host.argtypes = [v, ctypes.POINTER(Batch), ctypes.POINTER(Result)]
    lib.t2b_estep_batch_device.argtypes = [v, ctypes.POINTER(Batch), ctypes.POINTER(Result), v]
    lib.t2b_estep_submit_host.argtypes = [v, ctypes.POINTER(Batch), ctypes.POINTER(Result),
                                          ctypes.POINTER(ctypes.c_longlong)]
    lib.t2b_estep_wait.argtypes = [v, ctypes.c_longlong]
    lib.t2b_reconstruct_divide.argtypes = [v, i, v]
    lib.t2b_reconstruct_divide_noalloc.argtypes = [v, v, i, i, i, i, i, i, i, v, v]
    lib.t2b_project.argtypes = [v, i, v, i, i, v]
    lib.t2b_debug_coarse_diff2.argtypes = [v, i, v]
    lib.t2b_debug_fine.argtypes = [v, i, v, v, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    lib.t2b_debug_proposals.argtypes = [v, i, v, v, ctypes.POINTER(ctypes.c_int)]
    lib.t2b_debug_weights.argtypes = [v, i, v, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    lib.t2b_debug_selection.argtypes = [v, i, ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.t2b_last_stage_ms.argtypes = [v, v, i]
    lib.t2b_last_launch_count.argtypes = [v, ctypes.POINTER(i)]
    lib.t2b_stage_timing.argtypes = [v, i]
    lib.t2b_sampling.argtypes = [i, i, ctypes.c_double, i, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double] + [ctypes.POINTER(i)] * 5 + [v] * 6
    lib.t2b_proposal_train.argtypes = [v, ctypes.POINTER(ProposalTrainConfig), ctypes.POINTER(ProposalReport)]
    lib.t2b_proposal_enable.argtypes = [v, i, i, i, ctypes.c_double]
    lib.t2b_proposal_params.argtypes = [v, v, v, ctypes.POINTER(ctypes.c_longlong)]
    lib.t2b_proposal_features.argtypes = [v, ctypes.POINTER(Batch), v]
    lib.t2b_proposal_logits.argtypes = [v, v, i, v]
    lib.t2b_proposal_grad.argtypes = [v, v, v, v, i, ctypes.POINTER(ctypes.c_double), v]
    lib.t2b_prep_configure.argtypes = [v, ctypes.POINTER(PrepConfig)]
    lib.t2b_autotune.argtypes = [v, ctypes.POINTER(Batch), ctypes.POINTER(TuneReport)]
    lib.t2b_reconstruct.argtypes = [v, i, ctypes.POINTER(ReconConfig), v]
    ll = ctypes.c_longlong
    lib.t2b_mrc_info.argtypes = [c] + [ctypes.POINTER(i)] * 4 + [ctypes.POINTER(ctypes.c_double)]
    lib.t2b_mrc_read.argtypes = [c, ll, ll, v]
    lib.t2b_mrc_write.argtypes = [c, v, i, i, i, ctypes.c_double]
    lib.t2b_star_open.argtypes = [c, c, ctypes.POINTER(v)]
    lib.t2b_star_shape.argtypes = [v, ctypes.POINTER(ll), ctypes.POINTER(i)]
    lib.t2b_star_label.argtypes = [v, i, c, i]
    lib.t2b_star_column.argtypes = [v, c, v]
    lib.t2b_star_value.argtypes = [v, c, ll, c, i]
    lib.t2b_star_close.argtypes = [v]
    lib.t2b_star_close.restype = None
    lib.t2b_star_write.argtypes = [c, c, i, ctypes.POINTER(c), ll, v, i]
    lib.t2b_fsc_halves.argtypes = [v, i, i, i, v]
    lib.t2b_update_ssnr.argtypes = [v, i, ctypes.POINTER(SsnrConfig), v, v, v, v]
    lib.t2b_tune_set.argtypes = [v, ctypes.POINTER(TuneReport)]
    lib.t2b_prep_batch_host.argtypes = [v, ctypes.POINTER(PrepBatch), ctypes.POINTER(PrepOut)]
    lib.t2b_prep_batch_device.argtypes = [v, ctypes.POINTER(PrepBatch), ctypes.POINTER(PrepOut), v]


_setup_prototypes()


def _check(code):
    if code != T2B_OK:
        raise T2BError(code, lib.t2b_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def version():
    return lib.t2b_version().decode()


def point_group(group):
    """t2b_point_group: the operators of a point group other than the identity, an
    (n, 3, 3) array (SymList after read_sym_file, src/symmetries.cpp:51-191)."""
    n = ctypes.c_int(0)
    _check(lib.t2b_point_group(group.encode(), None, 0, ctypes.byref(n)))
    m = np.zeros((max(n.value, 1), 3, 3))
    _check(lib.t2b_point_group(group.encode(), _ptr(m), n.value, ctypes.byref(n)))
    return m[:n.value]


# ------------------------------------------------------------------ on-disk formats
def mrc_info(path):
    """(nx, ny, nz, mode, pixel size) of an MRC file (t2b_mrc_info)."""
    v = [ctypes.c_int() for _ in range(4)]
    px = ctypes.c_double()
    _check(lib.t2b_mrc_info(os.fsencode(path), *[ctypes.byref(x) for x in v], ctypes.byref(px)))
    return v[0].value, v[1].value, v[2].value, v[3].value, px.value


def read_mrc(path, first=0, count=None):
    """Sections [first, first + count) of an MRC stack as float32 (count, ny, nx)."""
    nx, ny, nz, _, _ = mrc_info(path)
    count = nz - first if count is None else count
    out = np.zeros((count, ny, nx), np.float32)
    _check(lib.t2b_mrc_read(os.fsencode(path), first, count, _ptr(out)))
    return out


def write_mrc(path, data, pixel_size):
    """Write (nz, ny, nx) or (ny, nx) float32 data as mode-2 MRC."""
    d = np.ascontiguousarray(data, np.float32)
    if d.ndim == 2:
        d = d[None]
    _check(lib.t2b_mrc_write(os.fsencode(path), _ptr(d), d.shape[2], d.shape[1], d.shape[0], float(pixel_size)))


class StarTable:
    """One data block of a STAR file (t2b_star_*): labels, text values, numeric columns."""

    def __init__(self, path, block=None):
        self._h = ctypes.c_void_p()
        _check(lib.t2b_star_open(os.fsencode(path), None if block is None else block.encode(), ctypes.byref(self._h)))
        rows, cols = ctypes.c_longlong(), ctypes.c_int()
        _check(lib.t2b_star_shape(self._h, ctypes.byref(rows), ctypes.byref(cols)))
        self.rows = rows.value
        buf = ctypes.create_string_buffer(256)
        self.labels = []
        for k in range(cols.value):
            _check(lib.t2b_star_label(self._h, k, buf, 256))
            self.labels.append(buf.value.decode())

    def column(self, label):
        out = np.zeros(self.rows)
        _check(lib.t2b_star_column(self._h, label.encode(), _ptr(out)))
        return out

    def value(self, label, row):
        buf = ctypes.create_string_buffer(4096)
        _check(lib.t2b_star_value(self._h, label.encode(), row, buf, 4096))
        return buf.value.decode()

    def strings(self, label):
        return [self.value(label, r) for r in range(self.rows)]

    def close(self):
        if self._h:
            lib.t2b_star_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_star(path, block, columns, append=False):
    """Write a numeric loop_ block: columns = {label: array of rows}."""
    labels = list(columns)
    vals = np.ascontiguousarray(np.stack([np.asarray(columns[k], np.float64) for k in labels], 1))
    arr = (ctypes.c_char_p * len(labels))(*[k.encode() for k in labels])
    _check(lib.t2b_star_write(os.fsencode(path), block.encode(), len(labels), arr, vals.shape[0], _ptr(vals),
                              int(append)))


def prep_params_from_star(particles, pixel_size, scale_correction=1.0):
    """Per-particle t2b_prep_batch parameters (n x 12) from a RELION particles block:
    offsets rlnOriginX/YAngst / pixel size (METADATA_XOFF/YOFF in pixels), priors (999: none),
    rlnNormCorrection, defocus U/V/angle, CTF B-factor, scale, phase shift."""
    n = particles.rows
    have = set(particles.labels)

    def col(name, default):
        return particles.column(name) if name in have else np.full(n, default)
    par = np.zeros((n, PREP_NPARAM))
    par[:, 0] = col("rlnOriginXAngst", 0.0) / pixel_size
    par[:, 1] = col("rlnOriginYAngst", 0.0) / pixel_size
    par[:, 2] = col("rlnOriginXPriorAngst", 999.0 * pixel_size) / pixel_size
    par[:, 3] = col("rlnOriginYPriorAngst", 999.0 * pixel_size) / pixel_size
    par[:, 4] = col("rlnNormCorrection", 1.0)
    par[:, 5] = col("rlnDefocusU", 0.0)
    par[:, 6] = col("rlnDefocusV", 0.0)
    par[:, 7] = col("rlnDefocusAngle", 0.0)
    par[:, 8] = col("rlnCtfBfactor", 0.0)
    par[:, 9] = col("rlnCtfScalefactor", 1.0)
    par[:, 10] = col("rlnPhaseShift", 0.0)
    par[:, 11] = scale_correction
    return par


def sampling(ref_dim, healpix_order, psi_step, adaptive_oversampling, offset_range_px,
             offset_step_px, pixel_size):
    """HealpixSampling-equivalent orientation / translation lists (C1, no perturbation).

    Returns a dict with eul_coarse (O x 9), eul_fine (O*R x 9), trans_px (T x 2),
    trans_px_fine (T*V x 2), trans_prior (T x 2, Angstrom), angles (O x 3) and
    the counts n_dir, n_psi, n_trans, nover_rot, nover_trans.
    """
    n = [ctypes.c_int() for _ in range(5)]
    args = (ref_dim, healpix_order, psi_step, adaptive_oversampling, offset_range_px,
            offset_step_px, pixel_size)
    _check(lib.t2b_sampling(*args, *[ctypes.byref(x) for x in n], *([None] * 6)))
    nd, npsi, nt, nr, nv = (x.value for x in n)
    o = nd * npsi
    out = dict(n_dir=nd, n_psi=npsi, n_trans=nt, nover_rot=nr, nover_trans=nv,
               eul_coarse=np.zeros((o, 9)), eul_fine=np.zeros((o * nr, 9)),
               trans_px=np.zeros((nt, 2)), trans_px_fine=np.zeros((nt * nv, 2)),
               trans_prior=np.zeros((nt, 2)), angles=np.zeros((o, 3)))
    _check(lib.t2b_sampling(*args, *[ctypes.byref(x) for x in n],
                            _ptr(out["eul_coarse"]), _ptr(out["eul_fine"]), _ptr(out["trans_px"]),
                            _ptr(out["trans_px_fine"]), _ptr(out["trans_prior"]), _ptr(out["angles"])))
    return out


def mresol_map(s):
    """Mresol of the window (src/ml_optimiser.cpp:5628-5660): ring index or -1."""
    xh = s // 2 + 1
    i = np.arange(s)[:, None]
    ip = np.where(i < xh, i, i - s)
    jp = np.arange(xh)[None, :]
    ires = np.rint(np.sqrt(ip * ip + jp * jp)).astype(np.int32)
    m = np.where((ires < xh) & ~((jp == 0) & (ip < 0)), ires, -1)
    return np.ascontiguousarray(m.reshape(-1), dtype=np.int32)


class EStep:
    """One E-step context on one GPU (MlDeviceBundle + MlOptimiserCuda)."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        _check(lib.t2b_create(device, ctypes.byref(self._h)))
        self._keep = []
        self._inflight = {}   # ticket -> the arrays a submitted host batch reads and writes
        self.cfg = None

    def close(self):
        if self._h:
            lib.t2b_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # AccProjector::setMdlDim + initMdl
    def set_projector(self, iclass, model, ref_dim, r_max, padding_factor):
        m = np.ascontiguousarray(model, dtype=np.complex64)
        if ref_dim == 3:
            zdim, ydim, xdim = m.shape
        else:
            ydim, xdim = m.shape
            zdim = 1
        _check(lib.t2b_projector_set(self._h, iclass, ref_dim, xdim, ydim, zdim, -(ydim // 2),
                                     -(zdim // 2) if ref_dim == 3 else 0, r_max, padding_factor,
                                     _ptr(m)))

    # AccBackprojector::setMdlDim + initMdl
    def init_backprojector(self, iclass, ref_dim, pad_size, r_max, padding_factor):
        xdim, ydim = pad_size // 2 + 1, pad_size
        zdim = pad_size if ref_dim == 3 else 1
        self._grid_shape = (zdim, ydim, xdim) if ref_dim == 3 else (ydim, xdim)
        if not hasattr(self, "_grid_dims"):
            self._grid_dims = {}
        self._grid_dims[iclass] = ref_dim
        _check(lib.t2b_backprojector_init(self._h, iclass, ref_dim, xdim, ydim, zdim, -(ydim // 2),
                                          -(zdim // 2) if ref_dim == 3 else 0, r_max, padding_factor))

    def clear_backprojector(self, iclass):
        _check(lib.t2b_backprojector_clear(self._h, iclass))

    # BackProjector::enforceHermitianSymmetry (before the reconstruction, once per iteration)
    def enforce_hermitian_symmetry(self, iclass):
        _check(lib.t2b_backprojector_enforce_hermitian(self._h, iclass))

    # BackProjector::applyPointGroupSymmetry
    def apply_point_group_symmetry(self, iclass, group):
        """t2b_backprojector_apply_symmetry: sum of the grid over the operators of a point
        group named as the reference's --sym ("C1", "C4", "D7", "D2h", "O", "I", "I3h" ...), in place."""
        _check(lib.t2b_backprojector_apply_symmetry(self._h, iclass, group.encode()))

    # BackProjector::applyHelicalSymmetry
    def apply_helical_symmetry(self, iclass, nr_asu, twist, rise, ori_size):
        """t2b_backprojector_apply_helical: sum of the grid over nr_asu helical units (twist in
        degrees, rise in pixels), in place."""
        _check(lib.t2b_backprojector_apply_helical(self._h, iclass, nr_asu, twist, rise, ori_size))

    # AccBackprojector::getMdlData
    def get_backprojector(self, iclass):
        shape = self._grid_shape
        re = np.zeros(shape, np.float32)
        im = np.zeros(shape, np.float32)
        w = np.zeros(shape, np.float32)
        _check(lib.t2b_backprojector_get(self._h, iclass, _ptr(re), _ptr(im), _ptr(w)))
        return re + 1j * im.astype(np.complex64), w

    def backprojector_device_ptrs(self, iclass):
        d, w = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib.t2b_backprojector_device_ptrs(self._h, iclass, ctypes.byref(d), ctypes.byref(w)))
        return d.value, w.value

    def configure(self, *, ori_size, current_size, ref_dim, nr_classes, samp, pdf_direction,
                  pdf_class, sigma2_offset, pixel_size, adaptive_fraction=0.999,
                  adaptive_oversampling=0, diff2_mode=DIFF2_PLAIN_FP32, max_batch=64,
                  fine_capacity=0, maximum_significants=-1, use_graph=1, data_vs_prior=None,
                  orientation_chunk=0):
        arrays = dict(
            eul_coarse=np.ascontiguousarray(samp["eul_coarse"], np.float64),
            eul_fine=np.ascontiguousarray(samp["eul_fine"], np.float64),
            trans_px=np.ascontiguousarray(samp["trans_px"], np.float64),
            trans_px_fine=np.ascontiguousarray(samp["trans_px_fine"], np.float64),
            trans_prior=np.ascontiguousarray(samp["trans_prior"], np.float64),
            pdf_direction=np.ascontiguousarray(pdf_direction, np.float64),
            pdf_class=np.ascontiguousarray(pdf_class, np.float64),
            mresol=mresol_map(current_size))
        if data_vs_prior is not None:
            arrays["data_vs_prior"] = np.ascontiguousarray(data_vs_prior, np.float64).reshape(
                nr_classes, ori_size // 2 + 1)
        c = Config()
        c.ori_size, c.current_size, c.ref_dim = ori_size, current_size, ref_dim
        c.nr_classes, c.n_dir, c.n_psi, c.n_trans = nr_classes, samp["n_dir"], samp["n_psi"], samp["n_trans"]
        c.adaptive_oversampling = adaptive_oversampling
        c.nover_rot = samp["nover_rot"] if adaptive_oversampling else 1
        c.nover_trans = samp["nover_trans"] if adaptive_oversampling else 1
        c.maximum_significants = maximum_significants
        c.diff2_mode, c.max_batch, c.use_graph = diff2_mode, max_batch, use_graph
        for k, a in arrays.items():
            setattr(c, k, _ptr(a))
        c.sigma2_offset, c.pixel_size, c.adaptive_fraction = sigma2_offset, pixel_size, adaptive_fraction
        c.fine_capacity = fine_capacity
        c.orientation_chunk = orientation_chunk
        _check(lib.t2b_configure(self._h, ctypes.byref(c)))
        self.cfg = dict(ori_size=ori_size, current_size=current_size, nr_classes=nr_classes,
                        n_dir=samp["n_dir"], n_psi=samp["n_psi"], n_trans=samp["n_trans"],
                        R=c.nover_rot, V=c.nover_trans, ovs=adaptive_oversampling,
                        max_batch=max_batch)
        return self.cfg

    def _result_arrays(self, n):
        cfg = self.cfg
        half = cfg["ori_size"] // 2 + 1
        K, nd = cfg["nr_classes"], cfg["n_dir"]
        return dict(
            min_diff2=np.zeros(n), sum_weight=np.zeros(n), sig_weight=np.zeros(n),
            coarse_sum_weight=np.zeros(n), coarse_sig_weight=np.zeros(n),
            nr_sign=np.zeros(n, np.int64), n_coarse_sig=np.zeros(n, np.int64), pmax=np.zeros(n),
            pose=np.zeros((n, 5), np.int32), wsum_norm=np.zeros(n), sumw=np.zeros(n),
            wsum_sigma2_offset=np.zeros(n), wsum_sigma2=np.zeros((n, half)),
            wsum_pdf_class=np.zeros((n, K)), wsum_pdf_dir=np.zeros((n, K * nd)),
            status=np.zeros(n, np.int32), audit_mass=np.zeros(n), learned=np.zeros(n, np.int32),
            wsum_scale_xa=np.zeros(n), wsum_scale_aa=np.zeros(n))

    # MlOptimiserCuda::doThreadExpectationSomeParticles for one batch (host buffers)
    def expectation(self, fimg, ctf, minvsigma2, scalars, fimg_nomask=None):
        fimg = np.ascontiguousarray(fimg, np.complex64)
        n = fimg.shape[0]
        arrs = [fimg, np.ascontiguousarray(ctf, np.float32), np.ascontiguousarray(minvsigma2, np.float32),
                np.ascontiguousarray(scalars, np.float64)]
        fnm = None if fimg_nomask is None else np.ascontiguousarray(fimg_nomask, np.complex64)
        b = Batch(n, 0, _ptr(arrs[0]), _ptr(fnm), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]))
        res = self._result_arrays(n)
        r = Result(*[_ptr(res[name]) for name, _ in Result._fields_])
        _check(lib.t2b_estep_batch_host(self._h, ctypes.byref(b), ctypes.byref(r)))
        return res

    # pipelined host batches: submit returns a ticket at once; the batch's arrays (inputs
    # and the returned result dict) must stay alive until wait(ticket) returns
    def expectation_submit(self, fimg, ctf, minvsigma2, scalars, fimg_nomask=None, out=None):
        fimg = np.ascontiguousarray(fimg, np.complex64)
        n = fimg.shape[0]
        arrs = [fimg, np.ascontiguousarray(ctf, np.float32), np.ascontiguousarray(minvsigma2, np.float32),
                np.ascontiguousarray(scalars, np.float64)]
        fnm = None if fimg_nomask is None else np.ascontiguousarray(fimg_nomask, np.complex64)
        b = Batch(n, 0, _ptr(arrs[0]), _ptr(fnm), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]))
        res = self._result_arrays(n) if out is None else out
        r = Result(*[_ptr(res[name]) for name, _ in Result._fields_])
        t = ctypes.c_longlong(-1)
        _check(lib.t2b_estep_submit_host(self._h, ctypes.byref(b), ctypes.byref(r), ctypes.byref(t)))
        self._inflight[t.value] = (arrs, fnm, res)
        return t.value, res

    def wait(self, ticket=-1):
        _check(lib.t2b_estep_wait(self._h, ticket))
        for k in [k for k in self._inflight if ticket < 0 or k <= ticket]:
            del self._inflight[k]

    # device-resident variant: arguments are objects with .data_ptr() (e.g. torch tensors)
    def expectation_device(self, n, fimg_ptr, ctf_ptr, minv_ptr, scal_ptr, result_ptrs, stream=0,
                           fimg_nomask_ptr=None):
        b = Batch(n, 0, fimg_ptr, fimg_nomask_ptr, ctf_ptr, minv_ptr, scal_ptr)
        r = Result(*[result_ptrs.get(name) for name, _ in Result._fields_])
        _check(lib.t2b_estep_batch_device(self._h, ctypes.byref(b), ctypes.byref(r),
                                          ctypes.c_void_p(stream)))

    # ---------------------------------------------- M-step reconstruction
    def reconstruct(self, iclass, ori_size, tau2=None, tau2_fudge=1.0, minres_map=0, gridding_iter=0, normalise=1.0):
        """t2b_reconstruct: the real-space map (ori_size^3, or ori_size^2 of a 2D class; FP64) of grid `iclass`;
        gridding_iter > 0: the gridding iterations (--dont_skip_gridding) with the class's sum of weights
        `normalise`."""
        t = None if tau2 is None else np.ascontiguousarray(tau2, np.float64)
        cfg = ReconConfig(ori_size, 0 if t is None else 1, minres_map, gridding_iter, tau2_fudge, _ptr(t), normalise)
        vol = np.zeros((ori_size,) * getattr(self, "_grid_dims", {}).get(iclass, 3))
        _check(lib.t2b_reconstruct(self._h, iclass, ctypes.byref(cfg), _ptr(vol)))
        return vol

    def fsc_halves(self, grid_a, grid_b, ori_size):
        """t2b_fsc_halves: down-sampled FSC of two grids (ori_size/2+1)."""
        f = np.zeros(ori_size // 2 + 1)
        _check(lib.t2b_fsc_halves(self._h, grid_a, grid_b, ori_size, _ptr(f)))
        return f

    def update_ssnr(self, iclass, ori_size, tau2, tau2_fudge=1.0, fsc=None, avgctf2=None,
                    is_whole_instead_of_half=False):
        """t2b_update_ssnr: returns (tau2, sigma2, data_vs_prior, fourier_coverage)."""
        nb = ori_size // 2 + 1
        t = np.array(tau2, np.float64).reshape(nb)
        f = None if fsc is None else np.ascontiguousarray(fsc, np.float64)
        a = None if avgctf2 is None else np.ascontiguousarray(avgctf2, np.float64)
        cfg = SsnrConfig(ori_size, f is not None, int(is_whole_instead_of_half), a is not None, tau2_fudge,
                         _ptr(f), _ptr(a))
        out = [np.zeros(nb) for _ in range(3)]
        _check(lib.t2b_update_ssnr(self._h, iclass, ctypes.byref(cfg), _ptr(t), *[_ptr(o) for o in out]))
        return (t, *out)

    # ---------------------------------------------- tile-shape autotuner
    def autotune(self, fimg, ctf, minvsigma2, scalars, fimg_nomask=None):
        """t2b_autotune on a host batch; returns the report as a dict (shapes and timings)."""
        fimg = np.ascontiguousarray(fimg, np.complex64)
        arrs = [np.ascontiguousarray(ctf, np.float32), np.ascontiguousarray(minvsigma2, np.float32),
                np.ascontiguousarray(scalars, np.float64)]
        fnm = None if fimg_nomask is None else np.ascontiguousarray(fimg_nomask, np.complex64)
        b = Batch(fimg.shape[0], 0, _ptr(fimg), _ptr(fnm), _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]))
        rep = TuneReport()
        _check(lib.t2b_autotune(self._h, ctypes.byref(b), ctypes.byref(rep)))
        return {k: (list(getattr(rep, k)) if isinstance(getattr(rep, k), ctypes.Array) else getattr(rep, k))
                for k, _ in TuneReport._fields_}

    def tune_set(self, diff2_tn=256, diff2_group=16, fine_ctas_per_sm=4, wsum_ctas_per_sm=4, project_pixels=256,
                 project_orients=1):
        """t2b_tune_set: install tile shapes (the defaults are the untuned ones)."""
        rep = TuneReport(diff2_tn=diff2_tn, diff2_group=diff2_group, fine_ctas_per_sm=fine_ctas_per_sm,
                         wsum_ctas_per_sm=wsum_ctas_per_sm, project_pixels=project_pixels,
                         project_orients=project_orients)
        _check(lib.t2b_tune_set(self._h, ctypes.byref(rep)))

    # ---------------------------------------------- image preparation
    def configure_prep(self, *, image_size, current_size, max_batch, sigma2_noise, pixel_size, mask_radius, **kw):
        """t2b_prep_configure (getFourierTransformsAndCtfs state of one optics group)."""
        opts = dict(PREP_DEFAULTS)
        unknown = set(kw) - set(opts)
        if unknown:
            raise TypeError(f"unknown image-preparation settings: {sorted(unknown)}")
        opts.update(kw)
        sig = np.ascontiguousarray(sigma2_noise, np.float64)
        self._prep_keep = sig
        c = PrepConfig(image_size=image_size, current_size=current_size, max_batch=max_batch,
                       n_sigma2=sig.size, sigma2_noise=_ptr(sig), pixel_size=pixel_size, mask_radius=mask_radius,
                       **opts)
        _check(lib.t2b_prep_configure(self._h, ctypes.byref(c)))
        self.prep_cfg = dict(image_size=image_size, current_size=current_size, max_batch=max_batch,
                             sigma2_noise=sig.copy(), pixel_size=pixel_size, mask_radius=mask_radius, **opts)
        return self.prep_cfg

    def prepare_images(self, images, params, part_id=None):
        """t2b_prep_batch_host: real-space images (n, N, N) and per-particle
        parameters (n, 12) -> dict(fimg, fimg_nomask, ctf, minvsigma2, scalars, power)."""
        pc = self.prep_cfg
        N, s = pc["image_size"], pc["current_size"]
        img = np.ascontiguousarray(images, np.float32)
        n = img.shape[0]
        par = np.ascontiguousarray(params, np.float64).reshape(n, PREP_NPARAM)
        pid = None if part_id is None else np.ascontiguousarray(part_id, np.int64)
        P = s * (s // 2 + 1)
        out = dict(fimg=np.zeros((n, P), np.complex64), fimg_nomask=np.zeros((n, P), np.complex64),
                   ctf=np.zeros((n, P), np.float32), minvsigma2=np.zeros((n, P), np.float32),
                   scalars=np.zeros((n, 8)), power=np.zeros((n, N // 2 + 1)))
        b = PrepBatch(n, 0, _ptr(img), _ptr(par), _ptr(pid))
        o = PrepOut(*[_ptr(out[k]) for k, _ in PrepOut._fields_])
        _check(lib.t2b_prep_batch_host(self._h, ctypes.byref(b), ctypes.byref(o)))
        return out

    def prepare_images_device(self, n, images_ptr, params_ptr, part_id_ptr, out_ptrs, stream=0):
        """t2b_prep_batch_device; pointers are device memory (ctypes.c_void_p)."""
        b = PrepBatch(n, 0, images_ptr, params_ptr, part_id_ptr)
        o = PrepOut(*[out_ptrs.get(k) for k, _ in PrepOut._fields_])
        _check(lib.t2b_prep_batch_device(self._h, ctypes.byref(b), ctypes.byref(o), ctypes.c_void_p(stream)))

    # ---------------------------------------------- learned orientation proposals
    def train_proposals(self, minvsigma2, n_train=200000, n_posterior=20000, n_val=1024, epochs=4, batch=256,
                        lr=3e-4, topk=64, rescore=0, seed=1, defocus=(10000., 30000.), astig=1000., voltage=300.,
                        cs=2.7, q0=0.1, max_shift=5.0, sigma_deg=5.0, alpha=3.0):
        """Train the proposal network on particles generated from the current
        references (t2b_proposal_train); returns the report as a dict."""
        mv = np.ascontiguousarray(minvsigma2, np.float32)
        c = ProposalTrainConfig(n_train, n_posterior, n_val, epochs, batch, lr, topk, rescore, seed, defocus[0],
                                defocus[1],
                                astig, voltage, cs, q0, max_shift, sigma_deg, alpha, _ptr(mv))
        rep = ProposalReport()
        _check(lib.t2b_proposal_train(self._h, ctypes.byref(c), ctypes.byref(rep)))
        out = {k: getattr(rep, k) for k, _ in ProposalReport._fields_ if k != "loss"}
        out["loss"] = list(rep.loss)[:min(epochs, 64)]
        return out

    def enable_proposals(self, topk=64, rescore=0, audit_every=50, audit_mass=0.999):
        _check(lib.t2b_proposal_enable(self._h, topk, rescore, audit_every, audit_mass))

    def disable_proposals(self):
        _check(lib.t2b_proposal_enable(self._h, 0, 0, 1, 1.0))

    def proposal_params(self, set_to=None):
        n = ctypes.c_longlong()
        _check(lib.t2b_proposal_params(self._h, None, None, ctypes.byref(n)))
        if set_to is not None:
            v = np.ascontiguousarray(set_to, np.float32)
            assert v.size == n.value
            _check(lib.t2b_proposal_params(self._h, None, _ptr(v), ctypes.byref(n)))
            return v
        out = np.zeros(n.value, np.float32)
        _check(lib.t2b_proposal_params(self._h, _ptr(out), None, ctypes.byref(n)))
        return out

    def proposal_features(self, fimg, ctf, minvsigma2):
        fimg = np.ascontiguousarray(fimg, np.complex64)
        ctf = np.ascontiguousarray(ctf, np.float32)
        mv = np.ascontiguousarray(minvsigma2, np.float32)
        n = fimg.shape[0]
        b = Batch(n, 0, _ptr(fimg), None, _ptr(ctf), _ptr(mv), None)
        out = np.zeros((n, 256), np.float32)
        _check(lib.t2b_proposal_features(self._h, ctypes.byref(b), _ptr(out)))
        return out

    def proposal_logits(self, imgs):
        imgs = np.ascontiguousarray(imgs, np.float32)
        cfg = self.cfg
        out = np.zeros((imgs.shape[0], cfg["nr_classes"] * cfg["n_dir"] * cfg["n_psi"]), np.float32)
        _check(lib.t2b_proposal_logits(self._h, _ptr(imgs), imgs.shape[0], _ptr(out)))
        return out

    def proposal_grad(self, imgs, tgt_oc, tgt_w):
        imgs = np.ascontiguousarray(imgs, np.float32)
        to = np.ascontiguousarray(tgt_oc, np.int32)
        tw = np.ascontiguousarray(tgt_w, np.float32)
        n = ctypes.c_longlong()
        _check(lib.t2b_proposal_params(self._h, None, None, ctypes.byref(n)))
        g = np.zeros(n.value, np.float32)
        loss = ctypes.c_double()
        _check(lib.t2b_proposal_grad(self._h, _ptr(imgs), _ptr(to), _ptr(tw), imgs.shape[0], ctypes.byref(loss),
                                     _ptr(g)))
        return loss.value, g

    def launch_count(self):
        k = ctypes.c_int()
        _check(lib.t2b_last_launch_count(self._h, ctypes.byref(k)))
        return k.value

    def stage_timing(self, on):
        _check(lib.t2b_stage_timing(self._h, 1 if on else 0))

    def stage_ms(self):
        ms = np.zeros(9, np.float32)
        _check(lib.t2b_last_stage_ms(self._h, _ptr(ms), 9))
        return ms

    def coarse_diff2(self, b):
        cfg = self.cfg
        out = np.zeros(cfg["nr_classes"] * cfg["n_dir"] * cfg["n_psi"] * cfg["n_trans"], np.float32)
        _check(lib.t2b_debug_coarse_diff2(self._h, b, _ptr(out)))
        return out

    def proposals(self, b):
        """Learned proposals of particle b in the last batch: (orientations, coarse diff2 kprop x n_trans)."""
        k = ctypes.c_int(0)
        _check(lib.t2b_debug_proposals(self._h, b, None, None, ctypes.byref(k)))
        prop = np.zeros(k.value, np.int32)
        d2 = np.zeros((k.value, self.cfg["n_trans"]), np.float32)
        _check(lib.t2b_debug_proposals(self._h, b, _ptr(prop), _ptr(d2), ctypes.byref(k)))
        return prop, d2

    def fine(self, b, cap=1 << 20):
        cfg = self.cfg
        cnt = ctypes.c_longlong()
        _check(lib.t2b_debug_fine(self._h, b, None, None, 0, ctypes.byref(cnt)))
        m = min(cnt.value, cap)
        pairs = np.zeros(max(m, 1), np.int64)
        d2 = np.zeros((max(m, 1), cfg["R"] * cfg["V"]), np.float32)
        _check(lib.t2b_debug_fine(self._h, b, _ptr(pairs), _ptr(d2), m, ctypes.byref(cnt)))
        return pairs[:m], d2[:m]

    def weights(self, b, cap=1 << 24):
        """Final-pass FP64 weights of particle b in the last batch (pairs x R*V, or one per pair)."""
        cnt = ctypes.c_longlong()
        _check(lib.t2b_debug_weights(self._h, b, None, 0, ctypes.byref(cnt)))
        m = min(cnt.value, cap)
        out = np.zeros(max(m, 1))
        _check(lib.t2b_debug_weights(self._h, b, _ptr(out), m, ctypes.byref(cnt)))
        return out[:m]

    def selection_path(self, b):
        """(coarse, fine) significance search of particle b: 2 one-CTA, 1 multi-kernel with the
        fast gather, 0 multi-kernel radix levels; fine is -1 without oversampling."""
        c, f = ctypes.c_int(), ctypes.c_int()
        _check(lib.t2b_debug_selection(self._h, b, ctypes.byref(c), ctypes.byref(f)))
        return c.value, f.value

    def reconstruct_divide(self, iclass):
        zdim, ydim, xdim = self._grid_shape
        ps = ydim
        out = np.zeros((ps, ps, ps // 2 + 1), np.complex128)
        _check(lib.t2b_reconstruct_divide(self._h, iclass, _ptr(out)))
        return out

    def project(self, iclass, eulers, current_size):
        e = np.ascontiguousarray(eulers, np.float64).reshape(-1, 9)
        P = current_size * (current_size // 2 + 1)
        out = np.zeros((e.shape[0], P), np.complex64)
        _check(lib.t2b_project(self._h, iclass, _ptr(e), e.shape[0], current_size, _ptr(out)))
        return out


# Reference-named wrappers (the names RELION's host code uses) ---------------
class AccProjector:
    """AccProjector (src/acc/acc_projector.h): setMdlDim + initMdl on a context."""

    def __init__(self, estep, iclass=0):
        self.estep, self.iclass = estep, iclass
        self._dims = None

    def setMdlDim(self, xdim, ydim, zdim, inity, initz, maxr, paddingFactor):
        self._dims = (xdim, ydim, zdim, inity, initz, maxr, paddingFactor)
        return True

    def initMdl(self, data):
        xdim, ydim, zdim, inity, initz, maxr, pad = self._dims
        ref_dim = 3 if zdim > 1 else 2
        shape = (zdim, ydim, xdim) if ref_dim == 3 else (ydim, xdim)
        self.estep.set_projector(self.iclass, np.asarray(data).reshape(shape), ref_dim, maxr, pad)


class AccBackprojector:
    """AccBackprojector (src/acc/acc_backprojector.h): grid on the device."""

    def __init__(self, estep, iclass=0):
        self.estep, self.iclass = estep, iclass

    def setMdlDim(self, xdim, ydim, zdim, inity, initz, max_r, paddingFactor):
        self._dims = (xdim, ydim, zdim, max_r, paddingFactor)
        return xdim * ydim * zdim * 12

    def initMdl(self):
        xdim, ydim, zdim, max_r, pad = self._dims
        self.estep.init_backprojector(self.iclass, 3 if zdim > 1 else 2, ydim, max_r, pad)

    def enforceHermitianSymmetry(self):
        self.estep.enforce_hermitian_symmetry(self.iclass)

    def applyPointGroupSymmetry(self, group):
        self.estep.apply_point_group_symmetry(self.iclass, group)

    def applyHelicalSymmetry(self, nr_helical_asu, helical_twist, helical_rise, ori_size):
        self.estep.apply_helical_symmetry(self.iclass, nr_helical_asu, helical_twist, helical_rise, ori_size)

    def getMdlData(self):
        data, w = self.estep.get_backprojector(self.iclass)
        return data.real.astype(np.float32), data.imag.astype(np.float32), w
