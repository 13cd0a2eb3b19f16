"""Tile-shape autotuner (t2b_autotune / t2b_tune_set): the shapes it picks come
from its candidate sets, its timings are real, the grids are left as they were,
and no shape changes what the E-step computes: coarse diff2, poses, nr_sign and
min_diff2 bit for bit; the FP64 weight sums to 1e-12 (they are accumulated from
per-block partial sums by atomics, whose order is never fixed)."""
import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu


def _run(es, P):
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    d2 = np.stack([es.coarse_diff2(b) for b in range(0, P["fimg"].shape[0], 5)])
    return res, d2


def _same(a, b):
    (ra, da), (rb, db) = a, b
    assert np.array_equal(da, db)
    assert np.array_equal(ra["pose"], rb["pose"])
    assert np.array_equal(ra["nr_sign"], rb["nr_sign"])
    assert np.array_equal(ra["min_diff2"], rb["min_diff2"])
    for k in ("sum_weight", "sig_weight", "coarse_sum_weight", "coarse_sig_weight", "pmax"):
        assert np.allclose(ra[k], rb[k], rtol=1e-12, atol=0), k


def test_autotune_picks_from_candidates_and_changes_no_value():
    pb = problems.build("refine_o1_ovs", n_particles=40, seed=17, diff2_mode=1)
    P = pb["parts"]
    es = pb["product"]()
    es.clear_backprojector(0)
    ref = _run(es, P)
    grid_before = es.get_backprojector(0)
    rep = es.autotune(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    print("autotune report:", rep)
    assert rep["diff2_tn"] in (256, 128) and rep["diff2_group"] in (4, 8, 16, 32)
    assert 1 <= rep["fine_ctas_per_sm"] <= 4 and 1 <= rep["wsum_ctas_per_sm"] <= 4
    assert rep["project_pixels"] in (128, 256, 512) and rep["project_orients"] in (1, 2, 4)
    assert all(t > 0 for t in rep["diff2_ms"] + rep["fine_ms"] + rep["wsum_ms"] + rep["project_ms"])
    i = (0 if rep["diff2_tn"] == 256 else 4) + (4, 8, 16, 32).index(rep["diff2_group"])
    assert rep["diff2_ms"][i] == min(rep["diff2_ms"])
    assert rep["project_ms"][3 * (128, 256, 512).index(rep["project_pixels"]) +
                             (1, 2, 4).index(rep["project_orients"])] == min(rep["project_ms"])
    # the tuning batches' backprojection was undone
    grid_after = es.get_backprojector(0)
    assert np.array_equal(grid_before[0], grid_after[0]) and np.array_equal(grid_before[1], grid_after[1])
    _same(_run(es, P), ref)
    es.close()


@pytest.mark.parametrize("shape", [dict(diff2_tn=128, diff2_group=4, fine_ctas_per_sm=1, wsum_ctas_per_sm=2,
                                        project_pixels=128, project_orients=4),
                                   dict(diff2_tn=256, diff2_group=32, fine_ctas_per_sm=3, wsum_ctas_per_sm=1,
                                        project_pixels=512, project_orients=2)],
                         ids=["n128_g4", "n256_g32"])
def test_installed_shapes_change_no_value(shape):
    """Explicit shapes, installed before t2b_configure (projection tables built with them)."""
    pb = problems.build("refine_o1_ovs", n_particles=40, seed=19, diff2_mode=1)
    P = pb["parts"]
    es = pb["product"]()
    ref = _run(es, P)
    proj_ref = es.project(0, pb["samp"]["eul_coarse"][:50], pb["s"])
    es.close()
    t2b, samp = pb["t2b"], pb["samp"]
    es2 = t2b.EStep(0)
    es2.tune_set(**shape)
    es2.set_projector(0, pb["maps"][0], 3, pb["r"], 2)
    es2.init_backprojector(0, 3, pb["pad_size"], pb["r"], 2)
    es2.configure(ori_size=pb["N"], current_size=pb["s"], ref_dim=3, nr_classes=1, samp=samp,
                  pdf_direction=np.ones((1, samp["n_dir"])) / samp["n_dir"], pdf_class=np.ones(1),
                  sigma2_offset=(3 * 2.0) ** 2, pixel_size=2.0, adaptive_oversampling=1, diff2_mode=1, max_batch=40)
    got = _run(es2, P)
    assert np.array_equal(es2.project(0, samp["eul_coarse"][:50], pb["s"]), proj_ref)
    _same(got, ref)
    es2.close()
