"""M-step reconstruction on the GPU (t2b_reconstruct, t2b_fsc_halves,
t2b_update_ssnr, t2b_backprojector_enforce_hermitian, t2b_backprojector_apply_symmetry,
t2b_backprojector_apply_helical) against the FP64 oracle (oracle/recon_oracle.py), on the
backprojection grids the E-step filled.

Tolerances: the map within 2e-5 of its largest value (the inverse 3D FFT is
FP32; the division before it and the sums after it are FP64); FSC and SSNR
arrays 1e-9 relative (FP64 sums in a different order)."""
import numpy as np
import pytest

import problems
import recon_oracle as ro

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def two_classes():
    pb = problems.build("refine_o2", n_particles=32, seed=23, nr_classes=2)
    P = pb["parts"]
    es = pb["product"]()
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    pb["es"] = es
    pb["grids"] = [es.get_backprojector(k) for k in range(2)]
    yield pb
    es.close()


def _map_close(got, ref):
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err <= 2e-5, err
    c = np.corrcoef(got.ravel(), ref.ravel())[0, 1]
    assert c >= 0.999999, c


@pytest.mark.parametrize("with_map", [False, True], ids=["plain", "map_tau2"])
def test_reconstruction_matches_oracle(two_classes, with_map):
    pb, es = two_classes, two_classes["es"]
    N, r = pb["N"], pb["r"]
    data, w = pb["grids"][0]
    tau2 = None
    if with_map:
        tau2 = np.random.default_rng(3).uniform(0.5, 2.0, N // 2 + 1) * np.mean(w)
    got = es.reconstruct(0, N, tau2=tau2, tau2_fudge=1.3, minres_map=2)
    ref = ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), r, 2, N, tau2=tau2, tau2_fudge=1.3,
                             minres_map=2)
    _map_close(got, ref)


def test_reconstruction_of_a_larger_grid_window_shrinks(t2b):
    """A grid whose pad_size (131) exceeds pad * ori_size (128): the transform is cut down."""
    pb = problems.build("refine_o2", n_particles=16, seed=29)
    P, samp = pb["parts"], pb["samp"]
    es = t2b.EStep(0)
    es.set_projector(0, pb["maps"][0], 3, pb["r"], 2)
    big_r = pb["N"] // 2
    es.init_backprojector(0, 3, 2 * (2 * big_r + 1) + 1, big_r, 2)
    es.configure(ori_size=pb["N"], current_size=pb["s"], ref_dim=3, nr_classes=1, samp=samp,
                 pdf_direction=np.ones((1, samp["n_dir"])) / samp["n_dir"], pdf_class=np.ones(1),
                 sigma2_offset=36.0, pixel_size=2.0, adaptive_oversampling=0, diff2_mode=0, max_batch=16)
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    data, w = es.get_backprojector(0)
    got = es.reconstruct(0, pb["N"])
    es.close()
    ref = ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), big_r, 2, pb["N"])
    _map_close(got, ref)


@pytest.mark.parametrize("name", ["refine_o2", "class2d"])
def test_hermitian_symmetry_matches_oracle(name):
    """t2b_backprojector_enforce_hermitian on an E-step grid, whose Friedel partners on the
    x = 0 plane differ (the backprojection puts each pixel on one of them), against the
    oracle's restatement of enforceHermitianSymmetry: each element is the same FP32 sum, so
    the grids are equal bit for bit; the reconstruction of the symmetrised grid matches the
    oracle's."""
    pb = problems.build(name, n_particles=16, seed=31)
    P = pb["parts"]
    es = pb["product"]()
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    data, w = es.get_backprojector(0)
    d0 = data[..., 0] if data.ndim == 3 else data[:, 0]
    assert np.max(np.abs(d0 - np.conj(d0[::-1, ::-1] if data.ndim == 3 else d0[::-1]))) > 0
    es.enforce_hermitian_symmetry(0)
    sd, sw = es.get_backprojector(0)
    rd, rw = ro.enforce_hermitian_symmetry(data, w)
    assert rd.dtype == np.complex64 and rw.dtype == np.float32
    assert np.array_equal(sd, rd) and np.array_equal(sw, rw)
    got = es.reconstruct(0, pb["N"])
    ref = ro.reconstruct_map(rd.astype(np.complex128), rw.astype(np.float64), pb["r"], 2, pb["N"])
    es.close()
    _map_close(got, ref)


@pytest.mark.parametrize("group", ["C3", "D2", "T", "I3", "C4v", "Oh"])
def test_point_group_symmetry_matches_oracle(group):
    """t2b_backprojector_apply_symmetry on the Hermitian-symmetrised grid of an E-step against
    the oracle's restatement of applyPointGroupSymmetry on the same FP32 grid: the coordinates
    are rounded as the reference rounds them, the reads and sums are FP64, so the device's
    FP32 result is the oracle's FP64 sum rounded once (rtol 1e-6); the symmetrised grid then
    reconstructs to the oracle's map."""
    pb = problems.build("refine_o2", n_particles=16, seed=37)
    P = pb["parts"]
    es = pb["product"]()
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.enforce_hermitian_symmetry(0)
    data, w = es.get_backprojector(0)
    es.apply_point_group_symmetry(0, group)
    gd, gw = es.get_backprojector(0)
    rd, rw = ro.apply_point_group_symmetry(data, w, ro.point_group(group), pb["r"], 2)
    for g, r in ((gd, rd), (gw, rw)):
        assert np.max(np.abs(g - r) / (np.abs(r) + 1e-9 * np.max(np.abs(r)))) <= 1e-6
    assert np.max(np.abs(gw - w)) > 0.1 * np.max(np.abs(w))
    got = es.reconstruct(0, pb["N"])
    es.close()
    ref = ro.reconstruct_map(gd.astype(np.complex128), gw.astype(np.float64), pb["r"], 2, pb["N"])
    _map_close(got, ref)


@pytest.mark.parametrize("nr_asu,twist,rise,group", [(5, -35.3, 4.7, "C1"), (2, 12.0, 0.0, "C1"), (3, 61.2, 2.9, "C3")])
def test_helical_symmetry_matches_oracle(nr_asu, twist, rise, group):
    """t2b_backprojector_apply_helical, then the point group, as MlOptimiser::maximization runs
    them on the Hermitian-symmetrised grid, against the oracle: 1e-6 relative per element (FP64
    coordinates, phases and sums, one FP32 rounding per step)."""
    pb = problems.build("refine_o2", n_particles=16, seed=43)
    P = pb["parts"]
    es = pb["product"]()
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.enforce_hermitian_symmetry(0)
    data, w = es.get_backprojector(0)
    es.apply_helical_symmetry(0, nr_asu, twist, rise, pb["N"])
    hd, hw = es.get_backprojector(0)
    mats, zsh = ro.helical_operators(nr_asu, twist, rise, pb["N"], 2)
    rd, rw = ro.apply_point_group_symmetry(data, w, mats, pb["r"], 2, zshift=zsh)
    for g, r in ((hd, rd), (hw, rw)):
        assert np.max(np.abs(g - r) / (np.abs(r) + 1e-9 * np.max(np.abs(r)))) <= 1e-6
    es.apply_point_group_symmetry(0, group)
    gd, gw = es.get_backprojector(0)
    es.close()
    rd2, rw2 = ro.apply_point_group_symmetry(hd, hw, ro.point_group(group), pb["r"], 2)
    for g, r in ((gd, rd2), (gw, rw2)):
        assert np.max(np.abs(g - r) / (np.abs(r) + 1e-9 * np.max(np.abs(r)))) <= 1e-6


def test_point_group_symmetry_identity_cases():
    """C1 leaves a 3D grid as it is, any group a 2D grid (the reference symmetrises 3D only);
    an unknown group (I5, not implemented by the reference either) is refused and the grid is
    left as it was; helical symmetry with one unit, or on a 2D grid, changes nothing."""
    t2b = problems.load_package()
    for name, group in (("refine_o2", "C1"), ("class2d", "O"), ("refine_o2", "I5"), ("refine_o2", "helix1"),
                        ("class2d", "helix5")):
        pb = problems.build(name, n_particles=8, seed=41)
        P = pb["parts"]
        es = pb["product"]()
        es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
        data, w = es.get_backprojector(0)
        if group == "I5":
            with pytest.raises(t2b.T2BError):
                es.apply_point_group_symmetry(0, group)
        elif group.startswith("helix"):   # one unit, or a 2D grid: unchanged
            es.apply_helical_symmetry(0, int(group[5:]), 20.0, 3.0, pb["N"])
        else:
            es.apply_point_group_symmetry(0, group)
        gd, gw = es.get_backprojector(0)
        es.close()
        assert np.array_equal(gd, data) and np.array_equal(gw, w)


def test_fsc_matches_oracle(two_classes):
    pb, es = two_classes, two_classes["es"]
    (d1, w1), (d2, w2) = pb["grids"]
    got = es.fsc_halves(0, 1, pb["N"])
    ref = ro.downsampled_fsc(d1.astype(np.complex128), w1.astype(np.float64), d2.astype(np.complex128),
                             w2.astype(np.float64), pb["r"], 2, pb["N"])
    assert np.allclose(got, ref, rtol=1e-9, atol=1e-12)
    same = es.fsc_halves(0, 0, pb["N"])
    assert np.allclose(same[:pb["r"] + 1], 1.0, atol=1e-12)


@pytest.mark.parametrize("with_fsc", [True, False], ids=["tau2_from_fsc", "keep_tau2"])
def test_ssnr_matches_oracle(two_classes, with_fsc):
    pb, es = two_classes, two_classes["es"]
    N, r = pb["N"], pb["r"]
    _, w = pb["grids"][0]
    nb = N // 2 + 1
    tau2 = np.random.default_rng(7).uniform(0.1, 1.0, nb) * np.mean(w)
    tau2[-3:] = 0.0
    fsc = np.clip(1.0 - np.linspace(0, 1.1, nb), -0.05, 1.0) if with_fsc else None
    got = es.update_ssnr(0, N, tau2, tau2_fudge=1.2, fsc=fsc)
    ref = ro.update_ssnr(w.astype(np.float64), r, 2, N, 1.2, tau2, fsc if with_fsc else np.zeros(nb),
                         update_tau2_with_fsc=with_fsc)
    for g, rr in zip(got, ref):
        assert np.allclose(g, rr, rtol=1e-9, atol=1e-14)


@pytest.fixture(scope="module")
def classes_2d():
    pb = problems.build("class2d", n_particles=24, seed=37, nr_classes=2)
    P = pb["parts"]
    es = pb["product"]()
    es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    pb["es"] = es
    pb["grids"] = [es.get_backprojector(k) for k in range(2)]
    yield pb
    es.close()


@pytest.mark.parametrize("with_map", [False, True], ids=["plain", "map_tau2"])
def test_2d_class_reconstruction_matches_oracle(classes_2d, with_map):
    pb, es = classes_2d, classes_2d["es"]
    N, r = pb["N"], pb["r"]
    for k in range(2):
        data, w = pb["grids"][k]
        assert w.ndim == 2
        tau2 = np.random.default_rng(9).uniform(0.5, 2.0, N // 2 + 1) * np.mean(w) if with_map else None
        got = es.reconstruct(k, N, tau2=tau2, tau2_fudge=2.0, minres_map=1)
        assert got.shape == (N, N)
        ref = ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), r, 2, N, tau2=tau2,
                                 tau2_fudge=2.0, minres_map=1)
        _map_close(got, ref)


def test_2d_fsc_and_ssnr_match_oracle(classes_2d):
    pb, es = classes_2d, classes_2d["es"]
    N, r = pb["N"], pb["r"]
    (d1, w1), (d2, w2) = pb["grids"]
    got = es.fsc_halves(0, 1, N)
    ref = ro.downsampled_fsc(d1.astype(np.complex128), w1.astype(np.float64), d2.astype(np.complex128),
                             w2.astype(np.float64), r, 2, N)
    assert np.allclose(got, ref, rtol=1e-9, atol=1e-12)
    nb = N // 2 + 1
    tau2 = np.random.default_rng(8).uniform(0.1, 1.0, nb) * np.mean(w1)
    g = es.update_ssnr(0, N, tau2, tau2_fudge=1.5, fsc=got)
    rr = ro.update_ssnr(w1.astype(np.float64), r, 2, N, 1.5, tau2, got)
    for a, b in zip(g, rr):
        assert np.allclose(a, b, rtol=1e-9, atol=1e-14)


@pytest.fixture(scope="module", params=["refine_o2", "class2d"])
def symmetric_grid(request):
    """A grid the E-step filled, Hermitian-symmetrised on the device (as the M-step receives
    it): 3D box 64 (pad_size 67, a prime) and 2D classes of box 48 (pad_size 51 = 3 x 17)."""
    pb = problems.build(request.param, n_particles=16, seed=31)
    P = pb["parts"]
    es = pb["product"]()
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.enforce_hermitian_symmetry(0)
    pb["es"] = es
    pb["grid"] = es.get_backprojector(0)
    pb["sumw"] = float(np.sum(res["sumw"]))
    yield pb
    es.close()


@pytest.mark.parametrize("with_map", [False, True], ids=["plain", "map_tau2"])
def test_gridding_reconstruction_matches_oracle(symmetric_grid, with_map):
    """--dont_skip_gridding: 10 iterations of the gridding weights (pad_size transforms of
    prime or composite odd length) before the windowed inverse transform, against the FP64
    oracle; the same tolerance as the skip-gridding path."""
    pb, es = symmetric_grid, symmetric_grid["es"]
    N, r = pb["N"], pb["r"]
    data, w = pb["grid"]
    tau2 = None
    if with_map:
        tau2 = np.random.default_rng(5).uniform(0.5, 2.0, N // 2 + 1) * np.mean(w)
    got = es.reconstruct(0, N, tau2=tau2, tau2_fudge=1.1, minres_map=1, gridding_iter=10, normalise=pb["sumw"])
    ref = ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), r, 2, N, tau2=tau2, tau2_fudge=1.1,
                             minres_map=1, gridding_iter=10, normalise=pb["sumw"])
    _map_close(got, ref)
    # and it is not the skip-gridding map
    skip = es.reconstruct(0, N, tau2=tau2, tau2_fudge=1.1, minres_map=1)
    assert np.max(np.abs(skip - got)) > 1e-3 * np.max(np.abs(got))


@pytest.mark.parametrize("r_max", [32, 64], ids=["pad131_prime", "pad259_7x37"])
def test_gridding_on_odd_boxes_from_a_written_grid(t2b, r_max):
    """The gridding iterations' transforms at pad sizes 131 (a prime: first-stage conjugate pairs)
    and 259 = 7 x 37 (37 in pairs, then the radix-7 register stage), on a seeded grid written into
    the library's device grid through its DLPack view (no E-step), against the oracle."""
    import torch
    import t2relion_b200.parallel as par
    ps = 2 * (2 * r_max + 1) + 1
    ori = 2 * r_max
    rng = np.random.default_rng(r_max)
    shape = (ps, ps, ps // 2 + 1)
    data = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    w = rng.uniform(0.5, 2.0, size=shape).astype(np.float32)
    es = t2b.EStep(0)
    es.init_backprojector(0, 3, ps, r_max, 2)
    nvox = int(np.prod(shape))
    d_ptr, w_ptr = es.backprojector_device_ptrs(0)
    dv = par.device_view(d_ptr, 2 * nvox, 0)
    wv = par.device_view(w_ptr, nvox, 0)
    dv.copy_(torch.from_numpy(np.ascontiguousarray(data).view(np.float32).reshape(-1)))
    wv.copy_(torch.from_numpy(w.reshape(-1)))
    torch.cuda.synchronize()
    del dv, wv
    gd, gw = es.get_backprojector(0)
    assert np.array_equal(gd, data) and np.array_equal(gw, w)
    got = es.reconstruct(0, ori, gridding_iter=2, normalise=3.0)
    es.close()
    ref = ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), r_max, 2, ori, gridding_iter=2,
                             normalise=3.0)
    _map_close(got, ref)
