"""The division entry point that allocates no device memory, through the C ABI.

t2b_reconstruct_divide_noalloc serves callers that cannot allocate device
memory (RELION's arena allocator has already reserved the GPU's free memory in
that process, and cudaMalloc/cudaFree would synchronise the whole device). It
must give the same FP64 result as t2b_reconstruct_divide, also on a second call
in a row (its fixed scratch array keeps the previous call's contents).
"""
import ctypes

import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu


def test_noalloc_division_matches_allocating_entry_point():
    import torch
    pb = problems.build("refine_o1_ovs", n_particles=8, seed=5)
    t2b = pb["t2b"]
    es = pb["product"]()
    P = pb["parts"]
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    assert np.all(res["status"] == 0)
    ref = es.reconstruct_divide(0)                 # allocating entry point
    data_ptr, w_ptr = es.backprojector_device_ptrs(0)
    ps, r = pb["pad_size"], pb["r"]
    stream = torch.cuda.Stream()
    for call in range(2):
        out = torch.full((ps, ps, ps // 2 + 1, 2), float("nan"), dtype=torch.float64, device="cuda")
        rc = t2b.lib.t2b_reconstruct_divide_noalloc(
            ctypes.c_void_p(data_ptr), ctypes.c_void_p(w_ptr), ps // 2 + 1, ps, ps, -(ps // 2), -(ps // 2),
            r, 2, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == t2b.T2B_OK, t2b.lib.t2b_last_error()
        stream.synchronize()
        got = out.cpu().numpy()
        got = got[..., 0] + 1j * got[..., 1]
        assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), call
    es.close()


def _noalloc(t2b, data_ptr, w_ptr, ps, r, stream):
    import torch
    out = torch.full((ps, ps, ps // 2 + 1, 2), float("nan"), dtype=torch.float64, device="cuda")
    rc = t2b.lib.t2b_reconstruct_divide_noalloc(
        ctypes.c_void_p(data_ptr), ctypes.c_void_p(w_ptr), ps // 2 + 1, ps, ps, -(ps // 2), -(ps // 2), r, 2,
        ctypes.c_void_p(out.data_ptr()), None if stream is None else ctypes.c_void_p(stream.cuda_stream))
    assert rc == t2b.T2B_OK, t2b.lib.t2b_last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    return got[..., 0] + 1j * got[..., 1]


def test_noalloc_larger_then_smaller_grid():
    """A grid of larger r_max, then the smaller one again on the legacy default stream
    (stream NULL): each call clears what the previous one left in the shared array."""
    import torch
    pb = problems.build("refine_o1_ovs", n_particles=8, seed=6)
    t2b, P, samp = pb["t2b"], pb["parts"], pb["samp"]
    small = pb["product"]()
    small.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    ref_small = small.reconstruct_divide(0)
    big_r = pb["N"] // 2 - 4
    big = t2b.EStep(0)
    big.set_projector(0, pb["maps"][0], 3, pb["r"], 2)
    ps_big = 2 * (2 * big_r + 1) + 1
    big.init_backprojector(0, 3, ps_big, big_r, 2)
    big.configure(ori_size=pb["N"], current_size=pb["s"], ref_dim=3, nr_classes=1, samp=samp,
                  pdf_direction=np.ones((1, samp["n_dir"])) / samp["n_dir"], pdf_class=np.ones(1),
                  sigma2_offset=36.0, pixel_size=2.0, adaptive_oversampling=1, diff2_mode=0, max_batch=8)
    big.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    ref_big = big.reconstruct_divide(0)
    stream = torch.cuda.Stream()
    got = _noalloc(t2b, *big.backprojector_device_ptrs(0), ps_big, big_r, stream)
    assert np.max(np.abs(got - ref_big)) <= 1e-12 * max(1.0, np.max(np.abs(ref_big)))
    got = _noalloc(t2b, *small.backprojector_device_ptrs(0), pb["pad_size"], pb["r"], None)
    assert np.max(np.abs(got - ref_small)) <= 1e-12 * max(1.0, np.max(np.abs(ref_small)))
    big.close()
    small.close()


def test_noalloc_rejects_r_max_beyond_limit():
    pb = problems.build("refine_o1_ovs", n_particles=2, seed=5)
    t2b = pb["t2b"]
    big = 2049
    ps = 2 * (2 * big + 1) + 1
    rc = t2b.lib.t2b_reconstruct_divide_noalloc(
        ctypes.c_void_p(1), ctypes.c_void_p(1), ps // 2 + 1, ps, ps, -(ps // 2), -(ps // 2), big, 2,
        ctypes.c_void_p(1), None)
    assert rc == t2b.T2B_ERR_ARG
    assert "T2B_NOALLOC_MAX_RMAX" in t2b.lib.t2b_last_error().decode()
