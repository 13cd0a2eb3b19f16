"""Parity with several classes: 3D refinement with 2 classes and 2D
classification (2D references, in-plane sampling, adaptive oversampling) with
3 classes, both diff2 modes, against the FP64 oracle."""
import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu

_ORACLE = {}


@pytest.fixture(scope="module", params=[("refine_o1_ovs", 2, 0), ("refine_o1_ovs", 2, 1),
                                        ("class2d", 3, 0), ("class2d", 3, 1)],
                ids=["3d-k2-plain", "3d-k2-splitbf16", "2d-k3-plain", "2d-k3-splitbf16"])
def run(request):
    name, K, mode = request.param
    pb = problems.build(name, n_particles=12, seed=13, nr_classes=K, diff2_mode=mode)
    es = pb["product"]()
    P = pb["parts"]
    pb["res"] = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    key = (name, K)
    if key not in _ORACLE:
        _ORACLE[key] = (pb["prob"].estep(pb["oparts"]), pb["prob"].grids())
    pb["ores"], pb["ogrids"] = _ORACLE[key]
    pb["es"] = es
    yield pb
    es.close()


def test_status(run):
    assert np.all(run["res"]["status"] == 0)
    assert run["ores"]["fails"] == 0


def test_coarse_diff2(run):
    es, prob, op = run["es"], run["prob"], run["oparts"]
    for b in range(3):
        ref, _ = prob.coarse_diff2(op, b)
        got = es.coarse_diff2(b).astype(np.float64)
        ok = ref >= 0
        assert np.array_equal(got < 0, ~ok)
        assert np.max(np.abs(got[ok] - ref[ok]) / np.abs(ref[ok])) <= 1e-5


def test_pose_and_class(run):
    same = np.all(run["res"]["pose"] == run["ores"]["pose"], axis=1)
    assert same.mean() >= 0.999, (run["res"]["pose"][~same], run["ores"]["pose"][~same])


def test_class_sums(run):
    res, ores = run["res"], run["ores"]
    assert np.allclose(res["wsum_pdf_class"].sum(1), res["sumw"], rtol=1e-9)
    assert np.allclose(res["wsum_pdf_class"], ores["wsum_pdf_class"], rtol=1e-3, atol=1e-6)


def test_grids_fsc_per_class(run):
    es = run["es"]
    od, ow = run["ogrids"]
    for k in range(run["K"]):
        data, w = es.get_backprojector(k)
        sh = problems.shells_of(data.shape)
        f = problems.fsc(data.reshape(-1), od[k].reshape(-1), sh, sh.max() + 1)
        assert np.all(f[1:2 * run["r"] + 1] >= 0.999), (k, f[:2 * run["r"] + 1])
