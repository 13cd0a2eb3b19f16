"""The chunked coarse pass (configurations whose projection tables do not fit on the device)
against the resident-table pass, through the C ABI.

Chunked, each batch projects one chunk of a class's coarse orientations at a time, splits it
into the split-BF16 operands and contracts it into the batch's diff2 rows; the fine pass and
the weighted sums interpolate their projections from the models.  Every diff2 is the same dot
product over the same contraction blocks and every projection the same FP64 interpolation, so
coarse and fine diff2, weights, poses and sums equal the resident pass's bit for bit; the
grids and the FP64 sums of weights differ only by the order of their atomic additions.  Chunks of 1,000 and 700 rows
over 2 classes: partial chunks, and chunks that end at a class boundary; and 2D references (60
psi per class in chunks of 40), whose models are read as one-voxel-deep 3D textures.
"""
import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,chunk", [("refine_o2", 1000), ("refine_o1_ovs", 700), ("class2d", 40)])
def test_chunked_equals_resident(name, chunk):
    pb = problems.build(name, n_particles=12, seed=43, nr_classes=2, diff2_mode=1, scale_correction=True)
    P = pb["parts"]
    out = {}
    for c in (0, chunk):
        es = pb["product"](orientation_chunk=c)
        res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
        d2 = [es.coarse_diff2(b) for b in range(3)]
        fine = [es.fine(b) for b in range(3)] if pb["ovs"] else None
        grids = [es.get_backprojector(k) for k in range(2)]
        es.close()
        out[c] = (res, d2, fine, grids)
    (r0, d0, f0, g0), (r1, d1, f1, g1) = out[0], out[chunk]
    assert np.all(r0["status"] == 0) and np.all(r1["status"] == 0)
    for a, b in zip(d0, d1):
        assert np.array_equal(a, b)
    if f0 is not None:
        for (pa, da), (pb_, db) in zip(f0, f1):
            assert np.array_equal(pa, pb_) and np.array_equal(da, db)
    for k in ("pose", "nr_sign", "n_coarse_sig", "min_diff2", "sig_weight", "coarse_sig_weight"):
        assert np.array_equal(r0[k], r1[k]), k
    # FP64 sums taken by atomics, whose order is not fixed: equal to the last bits
    for k in ("sum_weight", "coarse_sum_weight", "pmax"):
        assert np.allclose(r0[k], r1[k], rtol=1e-12, atol=0), k
    for k in ("sumw", "wsum_pdf_class", "wsum_pdf_dir", "wsum_sigma2_offset"):
        assert np.allclose(r0[k], r1[k], rtol=1e-10, atol=0), k
    # per-item sums over pixels taken by FP32 atomics in shared memory: their order is not fixed
    for k in ("wsum_norm", "wsum_sigma2", "wsum_scale_xa", "wsum_scale_aa"):
        assert np.allclose(r0[k], r1[k], rtol=1e-6, atol=1e-12 * np.abs(r0[k]).max()), k
    for (da, wa), (db, wb) in zip(g0, g1):
        assert np.max(np.abs(da - db)) <= 1e-5 * np.max(np.abs(da))
        assert np.max(np.abs(wa - wb)) <= 1e-5 * np.max(wa)


def test_chunked_refuses_plain_and_proposals(t2b):
    pb = problems.build("refine_o2", n_particles=4, seed=43, diff2_mode=0)
    with pytest.raises(t2b.T2BError) as e:
        pb["product"](orientation_chunk=1000)
    assert e.value.code == t2b.T2B_ERR_UNSUPPORTED
    pb = problems.build("refine_o2", n_particles=4, seed=43, diff2_mode=1)
    es = pb["product"](orientation_chunk=1000)
    with pytest.raises(t2b.T2BError) as e:
        es.train_proposals(pb["parts"]["minv"][0], n_train=1000, epochs=1)
    assert e.value.code == t2b.T2B_ERR_UNSUPPORTED
    es.close()
