"""Pins of the FP64 oracle against the reference's own known answers (CPU)."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT


def test_ctf_golden_value(oracle):
    # tests/ctf.cpp:5-9 of the reference: setValues(10000,12000,90,300,2.7,0.1,0,1,0), getCTF(10,10)
    v = oracle.ctf_value([10000.0, 12000.0, 90.0, 300.0, 2.7, 0.1, 0.0, 1.0, 0.0], 10.0, 10.0)
    assert v == pytest.approx(0.59154, abs=5e-6)


def test_ctf_image_matches_generator(oracle, synth):
    p = [15000.0, 14500.0, 33.0, 300.0, 2.7, 0.1, 0.0, 1.0, 0.0]
    a = oracle.ctf_image(p, 128, 1.3, 80)
    b = synth.ctf_image(p, 128, 1.3, 80)
    assert np.max(np.abs(a - b)) < 1e-6


def _ref_hp():
    path = os.path.join(ROOT, "oracle", "_ref", "libhp_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference HEALPix not built (needs the reference tree)")
    lib = ctypes.CDLL(path)
    lib.ref_hp_pix2zphi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]
    return lib


@pytest.mark.parametrize("order", [0, 1, 2, 3, 4])
def test_healpix_matches_reference(oracle, order):
    ref = _ref_hp()
    z, f = ctypes.c_double(), ctypes.c_double()
    for pix in range(12 * 4 ** order):
        ref.ref_hp_pix2zphi(order, pix, ctypes.byref(z), ctypes.byref(f))
        oz, of = oracle.healpix_pix2zphi(order, pix)
        assert (oz, of) == (z.value, f.value)


def test_shift_convention(oracle, synth):
    """diff2 of a particle made from the reference at the true pose is minimal there."""
    N, r, s = 32, 8, 16
    vol = synth.blob_volume(N, 10, seed=3)
    fmap = synth.fourier_map(vol, r)
    samp = dict(n_dir=1, n_psi=1, n_trans=3, nover_rot=1, nover_trans=1,
                eul_coarse=synth.euler_matrix(10., 40., 70.).reshape(1, 9), eul_fine=np.zeros((1, 9)),
                trans_px=np.array([[0., 0.], [1.5, -1.], [-2., 0.5]]), trans_px_fine=np.zeros((3, 2)),
                trans_prior=np.zeros((3, 2)))
    pr = oracle.Problem(ori_size=N, s=s, ref_dim=3, maps=[fmap], r_max=r, pad=2, samp=samp,
                        pdf_direction=np.ones((1, 1)), pdf_class=np.ones(1), sigma2_offset=100.,
                        pixel_size=1., adaptive_fraction=0.999, ovs=0, bp_pad_size=synth.pad_size(r), bp_r_max=r)
    parts = synth.make_particles(fmap, 1, ori_size=N, s=s, r_max=r, angpix=1., snr=1e6, seed=1, max_shift=0)
    # rebuild the particle at the sampled pose with shift (1.5, -1)
    A = samp["eul_coarse"].reshape(3, 3)
    proj = synth.project(fmap, A[None], s, r)[0]
    ky, kx = synth.window_coords(s)
    X = parts["ctf"][0] * proj * np.exp(2j * np.pi * (kx * 1.5 + ky * -1.0) / N)
    mres = synth.mresol(s)
    P = pr.particles(X[None], parts["ctf"], parts["minv"], parts["scalars"], mres)
    d2, mn = pr.coarse_diff2(P, 0)
    assert np.argmin(d2) == 1
    assert d2[1] == pytest.approx(parts["scalars"][0, 1] / 2, abs=1e-6 * abs(d2).max())


def test_oracle_projection_matches_numpy(oracle, synth):
    N, r, s = 32, 8, 16
    fmap = synth.fourier_map(synth.blob_volume(N, 10, seed=4), r)
    samp = dict(n_dir=1, n_psi=1, n_trans=1, nover_rot=1, nover_trans=1, eul_coarse=np.eye(3).reshape(1, 9),
                eul_fine=np.zeros((1, 9)), trans_px=np.zeros((1, 2)), trans_px_fine=np.zeros((1, 2)),
                trans_prior=np.zeros((1, 2)))
    pr = oracle.Problem(ori_size=N, s=s, ref_dim=3, maps=[fmap], r_max=r, pad=2, samp=samp,
                        pdf_direction=np.ones((1, 1)), pdf_class=np.ones(1), sigma2_offset=1., pixel_size=1.,
                        adaptive_fraction=0.999, ovs=0, bp_pad_size=synth.pad_size(r), bp_r_max=r)
    rng = np.random.default_rng(0)
    for _ in range(5):
        A = synth.euler_matrix(*rng.uniform(-180, 180, 3))
        a = pr.project(0, A)
        b = synth.project(fmap, A[None], s, r)[0]
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


def _ref_acc():
    path = os.path.join(ROOT, "oracle", "_ref", "libacc_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference CPU kernels not built (needs the reference tree)")
    lib = ctypes.CDLL(path)
    f, i, p = ctypes.c_float, ctypes.c_int, ctypes.c_void_p
    lib.ref_coarse_diff2.argtypes = [p, i, i, i, i, i, i, i, p, i, p, p, p, i, i, p, p, i, f, p]
    lib.ref_coarse_diff2.restype = i
    return lib


def test_coarse_diff2_matches_reference_cpu_kernel(oracle, synth):
    """FP64 oracle vs the reference's CpuKernels::diff2_coarse (FP32) on the same inputs.

    The reference kernel takes the CTF-divided image and corr = Minvsigma2 CTF^2
    (acc_coarse.h:309-346), which is the same diff2 as the oracle's
    sum 0.5 M |CTF P - shift X|^2; agreement to FP32 accumulation accuracy pins the
    oracle's projection, phase-shift and difference conventions to reference code.
    """
    import problems
    lib = _ref_acc()
    pb = problems.build("refine_o2", n_particles=2, seed=29)
    samp, prob, P = pb["samp"], pb["prob"], pb["parts"]
    fmap = pb["maps"][0]
    mz, my, mx = fmap.shape
    mdl = np.ascontiguousarray(fmap.view(np.float32))
    O, T = prob.O, prob.T
    sel = np.arange(0, O, 1)[:1024]
    eul = samp["eul_coarse"].reshape(-1, 3, 3)[sel]
    einv = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
    s, N = pb["s"], pb["N"]
    tx = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 0] / N, np.float32)
    ty = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 1] / N, np.float32)
    for b in range(2):
        ref_o, _ = prob.coarse_diff2(pb["oparts"], b)
        ref_o = ref_o.reshape(O, T)[sel]
        ctf = P["ctf"][b].astype(np.float64)
        X = P["fimg"][b].astype(np.complex128) / ctf
        re = np.ascontiguousarray(X.real, np.float32)
        im = np.ascontiguousarray(X.imag, np.float32)
        corr = np.ascontiguousarray(P["minv"][b] * ctf * ctf, np.float32)
        out = np.zeros((len(sel), T), np.float32)
        rc = lib.ref_coarse_diff2(mdl.ctypes.data, mx, my, mz, -(my // 2), -(mz // 2), pb["r"], 2,
                                  einv.ctypes.data, len(sel), re.ctypes.data, im.ctypes.data, corr.ctypes.data,
                                  s // 2 + 1, s, tx.ctypes.data, ty.ctypes.data, T,
                                  float(P["scalars"][b, 1] / 2), out.ctypes.data)
        assert rc == 0
        rel = np.abs(out.astype(np.float64) - ref_o) / np.abs(ref_o)
        assert np.max(rel) < 5e-6, np.max(rel)      # measured 5.7e-7
        assert np.median(rel) < 5e-7                 # measured 9.5e-8
        assert np.array_equal(np.argmin(out, axis=1), np.argmin(ref_o, axis=1))


def _small_problem(t2b, synth, oracle, scale=1.0, dvp=None, n=2, seed=5):
    N, r, s = 32, 8, 16
    fmap = synth.fourier_map(synth.blob_volume(N, 12, seed=seed), r)
    samp = t2b.sampling(3, 1, 15.0, 1, 2, 1, 2.0)
    parts = synth.make_particles(fmap, n, ori_size=N, s=s, r_max=r, angpix=2.0, snr=0.5, seed=seed,
                                 max_shift=2.0)
    parts["scalars"][:, 6] = scale
    pr = oracle.Problem(ori_size=N, s=s, ref_dim=3, maps=[fmap], r_max=r, pad=2, samp=samp,
                        pdf_direction=np.ones((1, samp["n_dir"])), pdf_class=np.ones(1), sigma2_offset=16.,
                        pixel_size=2.0, adaptive_fraction=0.999, ovs=1, bp_pad_size=synth.pad_size(r), bp_r_max=r,
                        data_vs_prior=dvp)
    return pr, parts, samp, synth.mresol(s)


def test_hoisted_diff2_equals_literal_form(t2b, synth, oracle):
    """The oracle's coarse and fine diff2 hoist the CTF-scaled reference and the shifted
    image out of the per-hypothesis loop; every value equals the reference's literal
    per-pixel form (src/ml_optimiser.cpp:7251-7272) bit for bit."""
    pr, parts, samp, mres = _small_problem(t2b, synth, oracle, scale=1.1)
    op = pr.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], mres)
    d2, _ = pr.coarse_diff2(op, 1)
    rng = np.random.default_rng(3)
    for o, t in zip(rng.integers(0, pr.O, 40), rng.integers(0, pr.T, 40)):
        assert d2[o * pr.T + t] == pr.diff2_literal(op, 1, 0, samp["eul_coarse"][o], samp["trans_px"][t])
    mask = np.zeros(pr.O * pr.T, np.uint8)
    mask[rng.integers(0, mask.size, 30)] = 1
    pairs, fd, _ = pr.fine_diff2(op, 1, mask)
    R, V = samp["nover_rot"], samp["nover_trans"]
    for q in range(0, len(pairs), 7):
        o, t = divmod(int(pairs[q]), pr.T)
        for r in range(R):
            for v in range(V):
                lit = pr.diff2_literal(op, 1, 0, samp["eul_fine"][o * R + r], samp["trans_px_fine"][t * V + v])
                assert fd[q, r * V + v] == lit


def test_scale_correction_sums_follow_the_scale(t2b, synth, oracle):
    """XA / AA are divided by scale_correction and its square (src/ml_optimiser.cpp:8859-8860):
    a particle whose CTF is halved while its scale doubles has the same diff2, weights and
    A = scale CTF P, so its XA halves and its AA quarters; rings with data_vs_prior <= 3 add
    nothing, and without data_vs_prior both sums are 0."""
    dvp = np.full((1, 17), 5.0)
    dvp[0, 5:9] = 1.0
    pa, parts, _, mres = _small_problem(t2b, synth, oracle, scale=1.0, dvp=dvp)
    ra = pa.estep(pa.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], mres), nthreads=1)
    pb, parts_b, _, _ = _small_problem(t2b, synth, oracle, scale=2.0, dvp=dvp)
    ctf_b = (parts_b["ctf"].astype(np.float64) / 2).astype(np.float32)
    assert np.array_equal(ctf_b.astype(np.float64) * 2, parts_b["ctf"].astype(np.float64))
    rb = pb.estep(pb.particles(parts_b["fimg"], ctf_b, parts_b["minv"], parts_b["scalars"], mres), nthreads=1)
    assert np.array_equal(ra["pose"], rb["pose"])
    assert np.all(ra["wsum_scale_aa"] > 0)
    assert np.allclose(rb["wsum_scale_xa"], ra["wsum_scale_xa"] / 2, rtol=1e-12)
    assert np.allclose(rb["wsum_scale_aa"], ra["wsum_scale_aa"] / 4, rtol=1e-12)
    pn, parts_n, _, _ = _small_problem(t2b, synth, oracle, scale=1.0, dvp=None)
    rn = pn.estep(pn.particles(parts_n["fimg"], parts_n["ctf"], parts_n["minv"], parts_n["scalars"], mres),
                  nthreads=1)
    assert np.all(rn["wsum_scale_xa"] == 0) and np.all(rn["wsum_scale_aa"] == 0)
    pz, parts_z, _, _ = _small_problem(t2b, synth, oracle, scale=1.0, dvp=np.zeros((1, 17)))
    rz = pz.estep(pz.particles(parts_z["fimg"], parts_z["ctf"], parts_z["minv"], parts_z["scalars"], mres),
                  nthreads=1)
    assert np.all(rz["wsum_scale_xa"] == 0) and np.all(rz["wsum_scale_aa"] == 0)


def test_wsum_stage_alone_reproduces_the_estep(t2b, synth, oracle):
    """orc_wsum_bp (the stage the device's weighted sums are checked against on the same
    weights) gives the E-step's own sums and grid when fed the E-step's final weights,
    rebuilt here from the oracle's fine pass and weights."""
    dvp = np.full((1, 17), 5.0)
    pa, parts, samp, mres = _small_problem(t2b, synth, oracle, scale=1.05, dvp=dvp, n=1)
    op = pa.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], mres)
    ra = pa.estep(op, nthreads=1)
    d2, mn = pa.coarse_diff2(op, 0)
    rc, w, sw, sig, _ = pa.weights(op, 0, 0, d2, np.arange(d2.size), mn)
    mask = (w >= sig).astype(np.uint8)
    pairs, fd, fmn = pa.fine_diff2(op, 0, mask)
    rc, wf, fsum, fsig, _ = pa.weights(op, 0, 1, fd.reshape(-1), np.repeat(pairs, pa.RV), fmn)
    pb, _, _, _ = _small_problem(t2b, synth, oracle, scale=1.05, dvp=dvp, n=1)
    o = pb.wsum_bp(op, 0, pairs, wf, fsum, fsig)
    for k in ("wsum_norm", "sumw", "wsum_sigma2_offset", "pmax", "wsum_scale_xa", "wsum_scale_aa"):
        assert o[k] == ra[k][0], k
    assert np.array_equal(o["pose"], ra["pose"][0])
    assert np.array_equal(o["wsum_sigma2"], ra["wsum_sigma2"][0])
    assert np.array_equal(pb.bp_data, pa.bp_data) and np.array_equal(pb.bp_weight, pa.bp_weight)


def _ref_stage_setup(b=0, seed=29):
    """refine_o1_ovs problem, the oracle's own final-pass hypotheses of particle b, and the
    reference kernels' shared operands (model, fine orientations, fine shift phases)."""
    import problems
    lib = _ref_acc()
    f, i, p, ll = ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong
    lib.ref_fine_diff2.argtypes = [p, i, i, i, i, i, i, i, p, i, p, p, p, i, i, p, p, i, f, i, p, p, p, p, ll, p]
    lib.ref_wavg.argtypes = [p, i, i, i, i, i, i, i, p, i, p, p, p, i, i, p, p, i, p, f, f, p, p, p]
    lib.ref_backproject.argtypes = [p, p, i, i, p, p, i, p, p, p, f, f, p, i, p, p, p, i, i, i, i, i, i, i]
    for fn in (lib.ref_fine_diff2, lib.ref_wavg, lib.ref_backproject):
        fn.restype = i
    dvp = np.full((1, 33), 6.0)
    dvp[0, 14:] = 1.0           # rings from 14 on out of the scale-correction sums
    pb = problems.build("refine_o1_ovs", n_particles=2, seed=seed)
    prob, op, samp, P = pb["prob"], pb["oparts"], pb["samp"], pb["parts"]
    d2, mn = prob.coarse_diff2(op, b)
    rc, w, sw, sig, _ = prob.weights(op, b, 0, d2, np.arange(d2.size), mn)
    pairs, fd, fmn = prob.fine_diff2(op, b, (w >= sig).astype(np.uint8))
    rc, wf, fsum, fsig, _ = prob.weights(op, b, 1, fd.reshape(-1), np.repeat(pairs, prob.RV), fmn)
    fmap = pb["maps"][0]
    N, s = pb["N"], pb["s"]
    tpf = samp["trans_px_fine"]
    op_ = dict(lib=lib, pb=pb, b=b, pairs=pairs, fd=fd, wf=wf, fsum=fsum, fsig=fsig, dvp=dvp,
               mdl=np.ascontiguousarray(fmap.view(np.float32)), mshape=fmap.shape,
               tx=np.ascontiguousarray(-2 * np.pi * tpf[:, 0] / N, np.float32),
               ty=np.ascontiguousarray(-2 * np.pi * tpf[:, 1] / N, np.float32), xh=s // 2 + 1, s=s)
    return op_


def _dense_weights(st):
    """The final weights as the reference's kernels take them: one row of every fine
    translation per fine orientation holding a significant hypothesis (0 elsewhere)."""
    pb, prob = st["pb"], st["pb"]["prob"]
    R, V, T = prob.S.nover_rot, prob.S.nover_trans, prob.T
    w = st["wf"].reshape(len(st["pairs"]), R, V)
    rows = {}
    for q, ih in enumerate(st["pairs"]):
        o, t = divmod(int(ih), T)
        for r in range(R):
            for v in range(V):
                if w[q, r, v] >= st["fsig"]:
                    rows.setdefault(o * R + r, np.zeros(T * V))[t * V + v] = w[q, r, v]
    rot = np.array(sorted(rows))
    return rot, np.ascontiguousarray(np.stack([rows[k] for k in rot]), np.float32)


def test_fine_diff2_matches_reference_cpu_kernel(oracle):
    """The oracle's fine pass against CpuKernels::diff2_fine_2D<REF3D> (FP32) over the same
    significant pairs, 8 rotations x 4 shifts each (the reference's FinePassWeights jobs)."""
    st = _ref_stage_setup()
    lib, pb, b = st["lib"], st["pb"], st["b"]
    prob, samp, P = pb["prob"], pb["samp"], pb["parts"]
    R, V, T = prob.S.nover_rot, prob.S.nover_trans, prob.T
    pairs = st["pairs"]
    eul = samp["eul_fine"].reshape(-1, 3, 3)
    einv = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
    nj = len(pairs) * R
    rot_idx, trans_idx = np.zeros(nj * V, np.uint64), np.zeros(nj * V, np.uint64)
    job_idx, job_num = np.zeros(nj, np.uint64), np.full(nj, V, np.uint64)
    for q, ih in enumerate(pairs):
        o, t = divmod(int(ih), T)
        for r in range(R):
            e0 = (q * R + r) * V
            job_idx[q * R + r] = e0
            rot_idx[e0:e0 + V] = o * R + r
            trans_idx[e0:e0 + V] = t * V + np.arange(V)
    ctf = P["ctf"][b].astype(np.float64)
    X = P["fimg"][b].astype(np.complex128) / ctf
    re, im = (np.ascontiguousarray(a, np.float32) for a in (X.real, X.imag))
    corr = np.ascontiguousarray(P["minv"][b] * ctf * ctf, np.float32)
    out = np.zeros(nj * V, np.float32)
    mz, my, mx = st["mshape"]
    rc = lib.ref_fine_diff2(st["mdl"].ctypes.data, mx, my, mz, -(my // 2), -(mz // 2), pb["r"], 2, einv.ctypes.data,
                            einv.shape[0], re.ctypes.data, im.ctypes.data, corr.ctypes.data, st["xh"], st["s"],
                            st["tx"].ctypes.data, st["ty"].ctypes.data, T * V, float(P["scalars"][b, 1] / 2), nj,
                            rot_idx.ctypes.data, trans_idx.ctypes.data, job_idx.ctypes.data, job_num.ctypes.data,
                            nj * V, out.ctypes.data)
    assert rc == 0
    ref = st["fd"].reshape(-1)
    rel = np.abs(out.astype(np.float64) - ref) / np.abs(ref)
    assert np.max(rel) < 5e-6, np.max(rel)
    assert np.array_equal(np.argmin(out.reshape(-1, R * V), 1), np.argmin(st["fd"], 1))


def test_weighted_sums_match_reference_cpu_kernel(oracle):
    """The oracle's sigma2 ring sums and scale-correction XA / AA against CpuKernels::wavg_ref3D
    (FP32, REFCTF) on the same final weights.  Rings 0-14: ring 16 holds the pixels on the
    projection circle, where the reference tests the rotated radius in floating point and the
    oracle the integer radius of the pixel (a documented convention of both paths)."""
    st = _ref_stage_setup()
    lib, pb, b = st["lib"], st["pb"], st["b"]
    prob, samp, P = pb["prob"], pb["samp"], pb["parts"]
    T, V = prob.T, prob.S.nover_trans
    rot, wd = _dense_weights(st)
    eul = samp["eul_fine"].reshape(-1, 3, 3)[rot]
    einv = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
    re, im = (np.ascontiguousarray(a, np.float32) for a in (P["fimg"][b].real, P["fimg"][b].imag))
    ctf = np.ascontiguousarray(P["ctf"][b] * P["scalars"][b, 6], np.float32)
    Pn = re.size
    parts, xa, aa = np.zeros(Pn, np.float32), np.zeros(Pn, np.float32), np.zeros(Pn, np.float32)
    mz, my, mx = st["mshape"]
    rc = lib.ref_wavg(st["mdl"].ctypes.data, mx, my, mz, -(my // 2), -(mz // 2), pb["r"], 2, einv.ctypes.data,
                      len(rot), re.ctypes.data, im.ctypes.data, ctf.ctypes.data, st["xh"], st["s"],
                      st["tx"].ctypes.data, st["ty"].ctypes.data, T * V, wd.ctypes.data, float(st["fsum"]), 1e-38,
                      parts.ctypes.data, xa.ctypes.data, aa.ctypes.data)
    assert rc == 0
    prob2 = oracle.Problem(ori_size=pb["N"], s=st["s"], ref_dim=3, maps=pb["maps"], r_max=pb["r"], pad=2,
                           samp=samp, pdf_direction=np.ones((1, samp["n_dir"])), pdf_class=np.ones(1),
                           sigma2_offset=36., pixel_size=2.0, adaptive_fraction=0.999, ovs=1,
                           bp_pad_size=pb["pad_size"], bp_r_max=pb["r"], data_vs_prior=st["dvp"])
    o = prob2.wsum_bp(pb["oparts"], b, st["pairs"], st["wf"], st["fsum"], st["fsig"])
    mres = pb["sy"].mresol(st["s"])
    ring = np.bincount(mres[mres >= 0], parts[mres >= 0].astype(np.float64), 33)
    rel = np.abs(ring[:15] - o["wsum_sigma2"][:15]) / o["wsum_sigma2"][:15]
    assert np.max(rel) < 1e-5, rel
    sel = (mres >= 0) & (st["dvp"][0][np.maximum(mres, 0)] > 3.)
    for k, arr in (("wsum_scale_xa", xa), ("wsum_scale_aa", aa)):
        v = float(np.sum(arr[sel].astype(np.float64)))
        assert abs(v - o[k]) <= 1e-5 * abs(o[k]), (k, v, o[k])


def test_backprojection_matches_reference_cpu_kernel(oracle, synth):
    """The oracle's backprojection (backproject2Dto3D) against CpuKernels::backprojectRef3D
    (FP32) on the same final weights, compared after enforceHermitianSymmetry (the x = 0 plane's
    Friedel choice is rounding noise in both).  Pixels the two paths treat differently by
    construction carry zero Minvsigma2 here: the duplicated x = 0 column of negative y (the
    CPU path skips it, src/backprojector.cpp:136-141; the accelerated kernels backproject
    it) and the rim the accelerated kernel's x < floor(sqrt(r^2 - y^2)) leaves out."""
    import recon_oracle as ro
    st = _ref_stage_setup()
    lib, pb, b = st["lib"], st["pb"], st["b"]
    prob, samp, P = pb["prob"], pb["samp"], pb["parts"]
    T, V = prob.T, prob.S.nover_trans
    s, xh, r = st["s"], st["xh"], pb["r"]
    ky, kx = synth.window_coords(s)
    minv = P["minv"][b].astype(np.float32).copy()
    rim = kx >= np.floor(np.sqrt(np.maximum(r * r - ky * ky, 0))).astype(int)
    minv[((kx == 0) & (ky < 0)) | rim] = 0.
    minv[0] = P["scalars"][b, 0]       # the DC term carries minvsigma2_dc in both
    rot, wd = _dense_weights(st)
    # inverted matrices, as the reference's weighted-sum setup builds them for the backprojection
    # (generateEulerMatrices(..., inverse = true), src/acc/acc_store_weight_sum.h:1041-1046)
    eul = samp["eul_fine"].reshape(-1, 3, 3)[rot]
    eul = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
    re, im = (np.ascontiguousarray(a, np.float32) for a in (P["fimg"][b].real, P["fimg"][b].imag))
    ctf = np.ascontiguousarray(P["ctf"][b], np.float32)
    ps = pb["pad_size"]
    gshape = (ps, ps, ps // 2 + 1)
    gr, gi, gw = (np.zeros(gshape, np.float32) for _ in range(3))
    rc = lib.ref_backproject(re.ctypes.data, im.ctypes.data, xh, s, st["tx"].ctypes.data, st["ty"].ctypes.data,
                             T * V, wd.ctypes.data, minv.ctypes.data, ctf.ctypes.data, 1e-38, float(st["fsum"]),
                             eul.ctypes.data, len(rot), gr.ctypes.data, gi.ctypes.data, gw.ctypes.data, r, 2,
                             ps // 2 + 1, ps, ps, -(ps // 2), -(ps // 2))
    assert rc == 0
    prob2 = pb["oracle_problem"]()
    sc = P["scalars"][b:b + 1].copy()
    op2 = prob2.particles(P["fimg"][b:b + 1], P["ctf"][b:b + 1], minv[None], sc, synth.mresol(s))
    prob2.wsum_bp(op2, 0, st["pairs"], st["wf"], st["fsum"], st["fsig"])
    od, ow = prob2.grids()
    od, ow = ro.enforce_hermitian_symmetry(od[0], ow[0])
    rd, rw = ro.enforce_hermitian_symmetry(gr.astype(np.float64) + 1j * gi, gw.astype(np.float64))
    assert np.max(np.abs(rd - od)) <= 1e-5 * np.max(np.abs(od)), np.max(np.abs(rd - od)) / np.max(np.abs(od))
    assert np.max(np.abs(rw - ow)) <= 1e-5 * np.max(ow), np.max(np.abs(rw - ow)) / np.max(ow)
