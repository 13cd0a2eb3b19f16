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
