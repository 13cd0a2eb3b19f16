"""Parity of the CUDA E-step (through the C ABI) with the FP64 oracle.

Tolerances: diff2 relative error <= 1e-5; the same max-weight orientation and
translation for >= 99.9 % of particles; map FSC >= 0.999 to Nyquist.  The FP64
weight / significance stages (coarse and fine) are checked exactly by feeding the
product's own diff2 to the oracle, and the weighted sums + backprojection by
feeding the product's own final weights to the oracle's stage.
"""
import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu

DIFF2_RTOL = 1e-5


_ORACLE = {}


# (problem, diff2 mode, scale correction on): the scale-correction sums and per-particle
# scales != 1 run on one single-pass and one oversampled case
@pytest.fixture(scope="module", params=[("refine_o2", 0, False), ("refine_o1_ovs", 0, True),
                                        ("refine_o2", 1, True), ("refine_o1_ovs", 1, False)],
                ids=["o2-plain", "o1ovs-plain-scale", "o2-splitbf16-scale", "o1ovs-splitbf16"])
def run(request):
    name, mode, scl = request.param
    pb = problems.build(name, diff2_mode=mode, scale_correction=scl)
    es = pb["product"]()
    P = pb["parts"]
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    pb["es"], pb["res"] = es, res
    key = (name, scl)
    if key not in _ORACLE:
        ores = pb["prob"].estep(pb["oparts"])
        data, w = pb["prob"].grids()
        _ORACLE[key] = (ores, (data.copy(), w.copy()))
    pb["ores"], pb["ogrids"] = _ORACLE[key]
    pb["scl"] = scl
    yield pb
    es.close()


def test_projection_table_matches_oracle(run):
    es, prob, samp = run["es"], run["prob"], run["samp"]
    idx = np.arange(0, samp["eul_coarse"].shape[0], 97)
    got = es.project(0, samp["eul_coarse"][idx], run["s"])
    for j, o in enumerate(idx):
        ref = prob.project(0, samp["eul_coarse"][o])
        assert np.max(np.abs(got[j] - ref)) <= 2e-6 * np.max(np.abs(ref))


def test_coarse_diff2_relative_error(run):
    es, prob, op = run["es"], run["prob"], run["oparts"]
    worst = 0.
    for b in range(4):
        ref, _ = prob.coarse_diff2(op, b)
        got = es.coarse_diff2(b).astype(np.float64)
        worst = max(worst, np.max(np.abs(got - ref) / np.abs(ref)))
    assert worst <= DIFF2_RTOL, worst


def test_status_ok(run):
    assert np.all(run["res"]["status"] == 0)
    assert run["ores"]["fails"] == 0


def test_pose_agreement(run):
    res, ores = run["res"], run["ores"]
    same = np.all(res["pose"] == ores["pose"], axis=1)
    assert same.mean() >= 0.999, (res["pose"][~same], ores["pose"][~same])


def test_weights_match_oracle_on_same_diff2(run):
    """FP64 weights + significance, checked on the product's own coarse diff2."""
    es, prob, op, res = run["es"], run["prob"], run["oparts"], run["res"]
    for b in range(4):
        d2 = es.coarse_diff2(b).astype(np.float64)
        ok = d2 >= 0
        mn = d2[ok].min()
        rc, w, sw, sig, ns = prob.weights(op, b, 0, d2, np.arange(d2.size), mn)
        assert rc == 0
        # the sum of up to K*O*T FP64 weights in another order: 1e-10; single weights 1e-12
        assert res["coarse_sum_weight"][b] == pytest.approx(sw, rel=1e-10)
        assert res["coarse_sig_weight"][b] == pytest.approx(sig, rel=1e-12)
        assert res["nr_sign"][b] == ns
        assert res["n_coarse_sig"][b] == int(np.sum(w >= sig))


def test_coarse_selection_path(run):
    """The dense coarse pass (K*O*T hypotheses, far above one CTA's 8192) is decided by
    the multi-kernel significance search."""
    es, prob = run["es"], run["prob"]
    assert run["K"] * prob.O * prob.T > 8192
    for b in range(run["res"]["status"].size):
        c, f = es.selection_path(b)
        assert c in (0, 1), (b, c)
        assert (f == -1) == (not run["ovs"])


def test_fine_weights_match_oracle_on_same_diff2(run):
    """FP64 fine-pass weights, sum and threshold, checked on the product's own fine diff2
    (exp_ipass == 1 of src/ml_optimiser.cpp:7770-7990)."""
    if not run["ovs"]:
        pytest.skip("single-pass configuration")
    es, prob, op, res = run["es"], run["prob"], run["oparts"], run["res"]
    RV = prob.RV
    for b in range(res["status"].size):
        pairs, d2 = es.fine(b)
        d2 = d2.astype(np.float64).reshape(-1)
        ih = np.repeat(pairs, RV)
        rc, w, sw, sig, _ = prob.weights(op, b, 1, d2, ih, d2[d2 >= 0].min())
        assert rc == 0
        assert res["sum_weight"][b] == pytest.approx(sw, rel=1e-10)
        assert res["sig_weight"][b] == pytest.approx(sig, rel=1e-12)
        pw = es.weights(b)
        assert pw.size == w.size
        assert np.allclose(pw, w, rtol=1e-12, atol=0)
        assert np.array_equal(pw >= res["sig_weight"][b], w >= sig)
        assert res["min_diff2"][b] == pytest.approx(d2[d2 >= 0].min(), rel=1e-7)


def test_wsum_bp_matches_oracle_on_same_weights(run):
    """Weighted sums and backprojection (storeWeightedSums, src/ml_optimiser.cpp:8153-8700;
    backproject2Dto3D, src/backprojector.cpp:55-230) on the product's own final weights: the
    oracle's FP64 stage against the device's.  FP64 sums of weights (sumw, pdf_class,
    pdf_direction, sigma2_offset, pmax): 1e-12.  Sums over pixels, FP32 within a work item
    (sigma2 rings, norm, scale-correction XA / AA): 1e-5 relative.  Grids (FP32 atomics):
    every voxel within 1e-5 of the grid's largest magnitude."""
    es, op, res = run["es"], run["oparts"], run["res"]
    prob2 = run["oracle_problem"]()
    worst = {}

    def upd(k, v):
        worst[k] = max(worst.get(k, 0.), float(v))
    for b in range(res["status"].size):
        pairs, _ = es.fine(b)
        wf = es.weights(b)
        o = prob2.wsum_bp(op, b, pairs, wf, res["sum_weight"][b], res["sig_weight"][b])
        for k in ("sumw", "wsum_sigma2_offset", "pmax"):
            upd(k, abs(res[k][b] - o[k]) / abs(o[k]))
        for k in ("wsum_pdf_class", "wsum_pdf_dir"):
            upd(k, np.max(np.abs(res[k][b] - o[k])) / np.max(np.abs(o[k])))
        assert np.array_equal(res["pose"][b], o["pose"]), (b, res["pose"][b], o["pose"])
        upd("wsum_norm", abs(res["wsum_norm"][b] - o["wsum_norm"]) / o["wsum_norm"])
        sig_o, sig_p = o["wsum_sigma2"], res["wsum_sigma2"][b]
        ring = sig_o > 1e-9 * sig_o.sum()
        upd("wsum_sigma2", np.max(np.abs(sig_p[ring] - sig_o[ring]) / sig_o[ring]))
        assert np.all(sig_p[~ring] <= 1e-8 * sig_o.sum())
        if run["scl"]:
            for k in ("wsum_scale_xa", "wsum_scale_aa"):
                upd(k, abs(res[k][b] - o[k]) / abs(o[k]))
        else:
            assert res["wsum_scale_xa"][b] == 0. and res["wsum_scale_aa"][b] == 0.
    for k in ("sumw", "wsum_sigma2_offset", "pmax", "wsum_pdf_class", "wsum_pdf_dir"):
        assert worst[k] <= 1e-12, (k, worst)
    for k in ("wsum_norm", "wsum_sigma2") + (("wsum_scale_xa", "wsum_scale_aa") if run["scl"] else ()):
        assert worst[k] <= 1e-5, (k, worst)
    od, ow = prob2.grids()
    for k in range(run["K"]):
        data, w = es.get_backprojector(k)
        ed = np.max(np.abs(data - od[k])) / np.max(np.abs(od[k]))
        ew = np.max(np.abs(w - ow[k])) / np.max(np.abs(ow[k]))
        assert ed <= 1e-5 and ew <= 1e-5, (ed, ew, worst)


def test_fine_pass_matches_oracle(run):
    if not run["ovs"]:
        pytest.skip("single-pass configuration")
    es, prob, op = run["es"], run["prob"], run["oparts"]
    for b in range(4):
        pairs, d2 = es.fine(b)
        mask = np.zeros(run["K"] * prob.O * prob.T, np.uint8)
        mask[pairs] = 1
        opairs, od2, _ = prob.fine_diff2(op, b, mask)
        assert np.array_equal(pairs, opairs)
        assert np.max(np.abs(d2 - od2) / np.abs(od2)) <= DIFF2_RTOL


def test_final_weights_close(run):
    res, ores = run["res"], run["ores"]
    assert np.allclose(res["min_diff2"], ores["min_diff2"], rtol=DIFF2_RTOL)
    assert np.allclose(res["pmax"], ores["pmax"], rtol=2e-2, atol=1e-3)
    # only the significant hypotheses are summed: adaptive_fraction < sum <= 1
    assert np.all(res["sumw"] > 0.999 - 1e-9) and np.all(res["sumw"] <= 1 + 1e-9)
    assert np.allclose(res["sumw"], ores["sumw"], rtol=1e-3)
    assert np.allclose(res["wsum_pdf_class"].sum(1), res["sumw"], rtol=1e-9)
    assert np.allclose(res["wsum_sigma2"].sum(1), res["wsum_norm"], rtol=1e-6)
    rel = np.abs(res["wsum_norm"] - ores["wsum_norm"]) / ores["wsum_norm"]
    assert np.median(rel) < 1e-3
    # the oracle's weights come from its own FP64 diff2: agreement at the weights' level
    rel = np.abs(res["wsum_sigma2_offset"] - ores["wsum_sigma2_offset"]) / ores["wsum_sigma2_offset"]
    assert np.median(rel) < 1e-2
    tot = np.abs(res["wsum_sigma2"] - ores["wsum_sigma2"]).sum(1) / ores["wsum_sigma2"].sum(1)
    assert np.median(tot) < 1e-3
    pd = np.abs(res["wsum_pdf_dir"] - ores["wsum_pdf_dir"]).sum(1)
    assert np.median(pd) < 1e-2
    if run["scl"]:
        for k in ("wsum_scale_xa", "wsum_scale_aa"):
            rel = np.abs(res[k] - ores[k]) / np.abs(ores[k])
            assert np.median(rel) < 1e-3, (k, rel)


def test_backprojection_fsc(run):
    es = run["es"]
    data, w = es.get_backprojector(0)
    od, ow = run["ogrids"]
    od, ow = od[0], ow[0]
    sh = problems.shells_of(data.shape)
    nsh = run["r"] * 2 + 1
    f = problems.fsc(data.reshape(-1), od.reshape(-1), sh, sh.max() + 1)
    assert np.all(f[1:nsh] >= 0.999), f[:nsh]
    assert np.linalg.norm(w - ow) / np.linalg.norm(ow) < 1e-2


def test_reconstruct_division_matches_oracle(run, oracle):
    es = run["es"]
    data, w = es.get_backprojector(0)
    got = es.reconstruct_divide(0)
    ref = oracle.reconstruct_divide(data.astype(np.complex128), w.astype(np.float64), run["r"], 2)
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_splitbf16_matches_plain_with_many_tiles_per_cta():
    """96 particles: 72 x 11 contraction tiles, several per persistent CTA."""
    pb = problems.build("refine_o2", n_particles=96, seed=21)
    P = pb["parts"]
    out = {}
    for mode in (0, 1):
        pb_mode = dict(pb)
        es = problems.build("refine_o2", n_particles=96, seed=21, diff2_mode=mode)["product"]()
        res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
        d2 = np.stack([es.coarse_diff2(b) for b in range(0, 96, 7)])
        out[mode] = (res, d2)
        es.close()
    (r0, d0), (r1, d1) = out[0], out[1]
    assert np.all(r0["status"] == 0) and np.all(r1["status"] == 0)
    assert np.max(np.abs(d1.astype(np.float64) - d0) / np.abs(d0)) <= 2 * DIFF2_RTOL
    assert np.mean(np.all(r0["pose"] == r1["pose"], axis=1)) >= 0.98


@pytest.mark.parametrize("name,maxsig", [("refine_o2", 40), ("refine_o1_ovs", 25), ("refine_o2", 3000)],
                         ids=["o2-maxsig40", "o1ovs-maxsig25", "o2-maxsig3000"])
def test_maximum_significants_matches_oracle(name, maxsig):
    """--maxsig: the coarse threshold is the weight of rank min(crossing, maxsig - 1)
    (src/ml_optimiser.cpp:7945-7966); the fine pass is unaffected."""
    pb = problems.build(name, n_particles=12, seed=41, diff2_mode=1, maxsig=maxsig)
    P = pb["parts"]
    es = pb["product"]()
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    ores = pb["prob"].estep(pb["oparts"])
    for b in range(4):
        d2 = es.coarse_diff2(b).astype(np.float64)
        mn = d2[d2 >= 0].min()
        rc, wts, sw, sig, ns = pb["prob"].weights(pb["oparts"], b, 0, d2, np.arange(d2.size), mn)
        assert rc == 0
        assert res["nr_sign"][b] == ns and ns <= maxsig
        assert res["coarse_sig_weight"][b] == pytest.approx(sig, rel=1e-12)
        assert res["n_coarse_sig"][b] == int(np.sum(wts >= sig))
    es.close()
    assert np.all(res["status"] == 0)
    assert np.all(res["nr_sign"] <= maxsig)
    same = np.all(res["pose"] == ores["pose"], axis=1)
    assert same.mean() >= 0.9, same.mean()
