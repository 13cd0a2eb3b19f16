"""Learned orientation proposals on the GPU, through the C ABI.

- feature images, the gradient of the training kernels and the tensor-core
  inference logits against the FP64 oracle (oracle/proposal_oracle.py);
- training on particles generated from the references, and what it gains over
  the initial network (the matched filter of the references' projections);
- the E-step with proposals against the full E-step (same poses, the
  posterior mass the audit measures), and the device-side fallback to the full
  coarse pass when the proposals miss posterior mass;
- the CUDA-graph device batch with proposals against the host batch.
"""
import ctypes

import numpy as np
import pytest

import problems
import proposal_oracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def o2():
    pb = problems.build("learn_o2", n_particles=48, seed=21, diff2_mode=1)
    es = pb["product"]()
    pb["es"] = es
    yield pb
    es.close()


def _KO(pb):
    return pb["samp"]["n_dir"] * pb["samp"]["n_psi"] * pb["K"]


def test_features_match_oracle(o2):
    P = o2["parts"]
    got = o2["es"].proposal_features(P["fimg"][:16], P["ctf"][:16], P["minv"][:16])
    ref = po.features(P["fimg"][:16], P["ctf"][:16].astype(np.float64), P["minv"][:16].astype(np.float64), o2["s"])
    assert np.max(np.abs(got - ref)) <= 2e-5 * np.max(np.abs(ref))


def _random_params(KO, seed):
    rng = np.random.default_rng(seed)
    L = po.layout(KO)
    th = (rng.standard_normal(L["total"]) * 0.03).astype(np.float32)
    return L, po.bf16(th).astype(np.float32)


def test_gradient_matches_oracle(o2):
    """Training kernels (SIMT FP32 on BF16 weights) vs the FP64 oracle's gradient."""
    es, KO = o2["es"], _KO(o2)
    L, th = _random_params(KO, 5)
    es.proposal_params(set_to=th)
    rng = np.random.default_rng(6)
    n = 12
    imgs = rng.standard_normal((n, 256)).astype(np.float32)
    to = np.full((n, 9), -1, np.int32)
    tw = np.zeros((n, 9), np.float32)
    for b in range(n):
        k = rng.integers(1, 5)
        to[b, :k] = rng.choice(KO, k, replace=False)
        w = rng.random(k)
        tw[b, :k] = w / w.sum()
    skip = np.zeros(KO, bool)
    loss, g = es.proposal_grad(imgs, to, tw)
    rloss, rg = po.loss_grad(th, imgs, to, tw, skip, KO)
    assert loss == pytest.approx(rloss, rel=1e-5)
    for name, size in (("wc1", 144), ("bc1", 16), ("wc2", 4608), ("bc2", 32), ("w1", 1024 * 2048), ("b1", 1024),
                       ("w2", 1024 * 1024), ("b2", 1024), ("w3", KO * 1024), ("b3", KO)):
        a = g[L[name]:L[name] + size].astype(np.float64)
        r = rg[L[name]:L[name] + size]
        err = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
        assert err <= 1e-4, (name, err)


def test_tensor_core_logits_match_oracle(o2):
    """Inference path (tcgen05, BF16 activations) vs the FP64 forward pass."""
    es, KO = o2["es"], _KO(o2)
    L, th = _random_params(KO, 7)
    es.proposal_params(set_to=th)
    rng = np.random.default_rng(8)
    imgs = rng.standard_normal((20, 256)).astype(np.float32)
    got = es.proposal_logits(imgs)
    ref, _ = po.forward(th, imgs, KO)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 2e-2, err
    # the ranked proposals agree
    for b in range(20):
        a = set(np.argsort(-got[b])[:64])
        r = set(np.argsort(-ref[b])[:64])
        assert len(a & r) >= 54


@pytest.fixture(scope="module")
def trained(o2):
    es = o2["es"]
    rep = es.train_proposals(o2["parts"]["minv"][0], n_train=40000, n_posterior=4096, n_val=512, epochs=4,
                             batch=256, lr=3e-4, topk=64, rescore=512, seed=3, max_shift=3.0)
    o2["report"] = rep
    return o2


def test_training_gains_over_initial_network(trained):
    """Held-out posterior mass in the top-64: the trained network against the
    matched filter it starts from, and with the low-resolution rescoring."""
    rep = trained["report"]
    print("proposal training report:", rep)
    assert rep["params"] > 10_000_000
    assert rep["loss"][-1] < rep["loss"][0]
    # the posterior mass the proposals miss shrinks at least fourfold with training
    assert 1.0 - rep["val_mass_trained"] <= 0.25 * (1.0 - rep["val_mass_init"]), rep
    assert rep["val_mass_rescored"] >= rep["val_mass_trained"], rep
    assert rep["val_frac_999_rescored"] >= 0.95, rep


def test_learned_estep_matches_full_estep(trained):
    es, P = trained["es"], trained["parts"]
    es.disable_proposals()
    full = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.enable_proposals(topk=64, rescore=512, audit_every=4, audit_mass=0.999)
    got = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.disable_proposals()
    assert np.all(got["status"] == 0)
    audited = got["audit_mass"] >= 0
    assert audited.sum() == len(audited) // 4
    assert np.all(got["learned"] == 1), got["audit_mass"][audited]
    assert np.all(got["audit_mass"][audited] >= 0.999)
    same = np.all(got["pose"] == full["pose"], axis=1)
    assert same.mean() >= 0.995, same.mean()


def test_audit_failure_falls_back_to_full_pass(o2):
    """Proposals that miss the posterior (all-zero network: the first orientations
    by index) make every audited batch run the full coarse pass."""
    es, P, KO = o2["es"], o2["parts"], _KO(o2)
    es.disable_proposals()
    full = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    saved = es.proposal_params()
    es.proposal_params(set_to=np.zeros(po.layout(KO)["total"], np.float32))
    es.enable_proposals(topk=64, audit_every=8, audit_mass=0.999)
    got = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    es.disable_proposals()
    es.proposal_params(set_to=saved)
    assert np.all(got["learned"] == 0)
    assert np.all(got["status"] == 0)
    assert np.array_equal(got["pose"], full["pose"])
    assert np.array_equal(got["nr_sign"], full["nr_sign"])
    assert np.allclose(got["sum_weight"], full["sum_weight"], rtol=1e-9)
    assert np.all(got["audit_mass"][got["audit_mass"] >= 0] < 0.999)


def test_graph_batch_with_proposals_matches_host(trained):
    import torch
    es, P = trained["es"], trained["parts"]
    n = 32
    es.enable_proposals(topk=64, rescore=512, audit_every=16, audit_mass=0.999)
    ref = es.expectation(P["fimg"][:n], P["ctf"][:n], P["minv"][:n], P["scalars"][:n])
    es.enable_proposals(topk=64, rescore=512, audit_every=16, audit_mass=0.999)  # restart the audit stream
    dev = torch.device("cuda")
    fimg = torch.from_numpy(np.ascontiguousarray(P["fimg"][:n]).view(np.float32)).to(dev)
    ctf = torch.from_numpy(np.ascontiguousarray(P["ctf"][:n])).to(dev)
    minv = torch.from_numpy(np.ascontiguousarray(P["minv"][:n])).to(dev)
    scal = torch.from_numpy(np.ascontiguousarray(P["scalars"][:n])).to(dev)
    host = es._result_arrays(n)
    tmap = {np.dtype("float64"): torch.float64, np.dtype("int64"): torch.int64, np.dtype("int32"): torch.int32}
    res = {k: torch.zeros(v.shape, dtype=tmap[v.dtype], device=dev) for k, v in host.items()}
    ptrs = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
    stream = torch.cuda.Stream()
    es.expectation_device(n, ctypes.c_void_p(fimg.data_ptr()), ctypes.c_void_p(ctf.data_ptr()),
                          ctypes.c_void_p(minv.data_ptr()), ctypes.c_void_p(scal.data_ptr()), ptrs,
                          stream=stream.cuda_stream)
    stream.synchronize()
    es.disable_proposals()
    got = {k: v.cpu().numpy() for k, v in res.items()}
    assert np.array_equal(got["learned"], ref["learned"])
    assert np.array_equal(got["pose"], ref["pose"])
    assert np.allclose(got["sum_weight"], ref["sum_weight"], rtol=1e-9)
    assert np.allclose(got["audit_mass"], ref["audit_mass"], rtol=1e-9)


def test_proposal_diff2_matches_full_pass(trained):
    """The restricted coarse pass (premultiplied proposal rows against the shared phase
    rows) against the full coarse pass at the same (orientation, translation): both
    split-BF16 contractions of the same sums, within 1e-5 of the diff2 scale."""
    es, P = trained["es"], trained["parts"]
    n = 16
    es.enable_proposals(topk=64, rescore=512, audit_every=1000, audit_mass=1e-6)
    got = es.expectation(P["fimg"][:n], P["ctf"][:n], P["minv"][:n], P["scalars"][:n])
    assert np.all(got["learned"] == 1)
    props = [es.proposals(b) for b in range(n)]
    es.disable_proposals()
    es.expectation(P["fimg"][:n], P["ctf"][:n], P["minv"][:n], P["scalars"][:n])
    T = trained["samp"]["n_trans"]
    worst = 0.0
    for b, (prop, d2) in enumerate(props):
        assert len(np.unique(prop)) == len(prop)
        full = es.coarse_diff2(b).reshape(-1, T)[prop]
        live = full > -998          # skipped orientations hold -999 in both
        assert np.array_equal(live, d2 > -998)
        scale = np.max(np.abs(full[live]))
        worst = max(worst, np.max(np.abs(d2[live] - full[live])) / scale)
    print("proposal diff2 vs full pass, max relative deviation:", worst)
    assert worst <= 1e-5


def test_audit_with_fewer_than_max_slots_graph_and_eager(trained):
    """Batches whose audited count is below the slot maximum run the narrower audit
    variant (each of the two launches gated on the device-side count): a stream of three
    32-particle batches audited every 20th particle (2, 2 and 1 audited) gives the same
    audit masses and poses replayed as graphs and launched one by one."""
    es, P = trained["es"], trained["parts"]
    n = 32
    runs = []
    for eager in (False, True):
        es.stage_timing(eager)
        es.enable_proposals(topk=64, rescore=512, audit_every=20, audit_mass=0.999)
        out = []
        for first in (0, 16, 0):
            sl = slice(first, first + n)
            out.append(es.expectation(P["fimg"][sl], P["ctf"][sl], P["minv"][sl], P["scalars"][sl]))
        runs.append(out)
    es.stage_timing(False)
    es.disable_proposals()
    counts = [int((r["audit_mass"] >= 0).sum()) for r in runs[0]]
    assert counts == [2, 2, 1], counts
    for a, b in zip(*runs):
        assert np.array_equal(a["learned"], b["learned"])
        assert np.array_equal(a["pose"], b["pose"])
        assert np.allclose(a["audit_mass"], b["audit_mass"], rtol=1e-9)
        assert np.all(a["audit_mass"][a["audit_mass"] >= 0] > 0.5)


def test_learned_coarse_selection_matches_oracle(trained):
    """The coarse significance of a learned batch (one CTA per particle over its
    proposals' hypotheses: weights, sum, candidates above the mass floor, threshold)
    against the FP64 oracle's weights and threshold on the same diff2 values."""
    es, P = trained["es"], trained["parts"]
    n = 16
    es.enable_proposals(topk=64, rescore=512, audit_every=1000, audit_mass=1e-6)
    res = es.expectation(P["fimg"][:n], P["ctf"][:n], P["minv"][:n], P["scalars"][:n])
    props = [es.proposals(b) for b in range(6)]
    es.disable_proposals()
    assert np.all(res["learned"] == 1)
    T = trained["samp"]["n_trans"]
    for b, (prop, d2) in enumerate(props):
        d2 = d2.astype(np.float64).ravel()
        ih = (prop[:, None].astype(np.int64) * T + np.arange(T)[None, :]).ravel()
        mn = d2[d2 >= 0].min()
        rc, wts, sw, sig, ns = trained["prob"].weights(trained["oparts"], b, 0, d2, ih, mn)
        assert rc == 0
        assert res["nr_sign"][b] == ns
        assert res["coarse_sig_weight"][b] == pytest.approx(sig, rel=1e-12)
        assert res["coarse_sum_weight"][b] == pytest.approx(sw, rel=1e-12)
        assert res["n_coarse_sig"][b] == int(np.sum(wts >= sig))


def test_low_snr_audit_falls_back_where_proposals_miss():
    """SNR 0.03 at box 64 (the noise level of the box-128 benchmark, where the posterior is
    broad): a network trained as above, 8-particle batches with one audited particle each.
    A batch whose audited particle keeps >= 0.999 of its posterior mass in its proposals stays
    on them; a batch where it does not runs the full coarse pass, and its results are then
    exactly the full E-step's.  At this noise level the fallback must fire in some batch, and
    the poses of the learned batches agree with the full E-step."""
    pb = problems.build("learn_o2_lowsnr", n_particles=64, seed=37, diff2_mode=1, max_batch=8)
    es, P = pb["product"](), pb["parts"]
    es.train_proposals(P["minv"][0], n_train=40000, n_posterior=4096, n_val=512, epochs=4, batch=256, lr=3e-4,
                       topk=64, rescore=512, seed=3, max_shift=3.0)
    fell, stayed, same, n = 0, 0, 0, 0
    for a in range(0, 64, 8):
        args = [P[k][a:a + 8] for k in ("fimg", "ctf", "minv", "scalars")]
        es.disable_proposals()
        full = es.expectation(*args)
        es.enable_proposals(topk=64, rescore=512, audit_every=8, audit_mass=0.999)
        got = es.expectation(*args)
        es.disable_proposals()
        assert np.all(got["status"] == 0)
        mass = got["audit_mass"][got["audit_mass"] >= 0]
        assert mass.size == 1
        if mass[0] < 0.999:
            fell += 1
            assert np.all(got["learned"] == 0)
            assert np.array_equal(got["pose"], full["pose"])
            assert np.array_equal(got["nr_sign"], full["nr_sign"])
            assert np.allclose(got["sum_weight"], full["sum_weight"], rtol=1e-9)
        else:
            stayed += 1
            assert np.all(got["learned"] == 1)
            same += int(np.all(got["pose"] == full["pose"], axis=1).sum())
            n += 8
    es.close()
    print(f"low-SNR audit: {fell} batches fell back, {stayed} stayed on the proposals")
    assert fell >= 1
    assert n == 0 or same / n >= 0.9
