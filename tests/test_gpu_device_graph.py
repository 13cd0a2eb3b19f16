"""Device-resident entry point with CUDA-graph replay vs the host entry point."""
import ctypes

import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "splitbf16"])
def test_graph_replay_matches_host_path(mode):
    import torch
    pb = problems.build("refine_o1_ovs", n_particles=12, seed=9, diff2_mode=mode)
    P = pb["parts"]
    es = pb["product"]()
    ref = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    n = P["fimg"].shape[0]
    dev = torch.device("cuda")
    fimg = torch.from_numpy(P["fimg"].view(np.float32)).to(dev)
    ctf = torch.from_numpy(P["ctf"]).to(dev)
    minv = torch.from_numpy(P["minv"]).to(dev)
    scal = torch.from_numpy(P["scalars"]).to(dev)
    host = es._result_arrays(n)
    res = {k: torch.zeros(v.shape, dtype={np.dtype("float64"): torch.float64, np.dtype("int64"): torch.int64,
                                          np.dtype("int32"): torch.int32}[v.dtype], device=dev)
           for k, v in host.items()}
    ptrs = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
    stream = torch.cuda.Stream()
    for rep in range(3):
        es.expectation_device(n, ctypes.c_void_p(fimg.data_ptr()), ctypes.c_void_p(ctf.data_ptr()),
                              ctypes.c_void_p(minv.data_ptr()), ctypes.c_void_p(scal.data_ptr()), ptrs,
                              stream=stream.cuda_stream)
        stream.synchronize()
        got = {k: v.cpu().numpy() for k, v in res.items()}
        assert np.all(got["status"] == 0)
        assert np.array_equal(got["pose"], ref["pose"]), rep
        assert np.array_equal(got["nr_sign"], ref["nr_sign"])
        for k in ("min_diff2", "sum_weight", "sig_weight", "pmax", "sumw"):
            assert np.allclose(got[k], ref[k], rtol=1e-9, atol=0), k
        # FP32 per-pixel terms accumulated by atomics in arbitrary order
        assert np.allclose(got["wsum_norm"], ref["wsum_norm"], rtol=1e-5, atol=0)
    # kernel nodes outside the conditional bodies (the selection's multi-kernel path)
    assert es.launch_count() >= 10
    es.close()


def test_pipelined_host_batches_match_synchronous_ones(t2b):
    """t2b_estep_submit_host / t2b_estep_wait: three batches of different sizes in flight
    at once (inputs copied while the previous batch computes, two staging slots) give
    the results and the backprojection of the same batches run one at a time."""
    pb = problems.build("refine_o1_ovs", n_particles=14, seed=12, diff2_mode=1)
    P = pb["parts"]
    es = pb["product"]()
    cuts = [(0, 6), (6, 9), (9, 14)]

    def part(a, b):
        return P["fimg"][a:b], P["ctf"][a:b], P["minv"][a:b], P["scalars"][a:b]

    es.clear_backprojector(0)
    sync = [es.expectation(*part(a, b)) for a, b in cuts]
    g_sync = [x.copy() for x in es.get_backprojector(0)]
    es.clear_backprojector(0)
    tickets = [es.expectation_submit(*part(a, b)) for a, b in cuts]
    assert [t for t, _ in tickets] == [tickets[0][0] + i for i in range(3)]
    es.wait(tickets[1][0])          # the first two are done, the third may still run
    for (t, got), ref in zip(tickets[:2], sync[:2]):
        assert np.array_equal(got["pose"], ref["pose"])
    es.wait()
    for (t, got), ref in zip(tickets, sync):
        assert np.all(got["status"] == 0)
        assert np.array_equal(got["pose"], ref["pose"])
        assert np.array_equal(got["nr_sign"], ref["nr_sign"])
        for k in ("min_diff2", "sum_weight", "sig_weight", "pmax", "sumw"):
            assert np.allclose(got[k], ref[k], rtol=1e-9, atol=0), k
        assert np.allclose(got["wsum_norm"], ref["wsum_norm"], rtol=1e-5, atol=0)
    for a, b in zip(es.get_backprojector(0), g_sync):
        assert np.allclose(a, b, rtol=1e-4, atol=1e-4 * np.max(np.abs(b)))
    with pytest.raises(t2b.T2BError):
        es.wait(tickets[-1][0] + 1)
    es.close()


def test_host_submissions_and_device_batch_are_ordered():
    """A device batch on the caller's stream, enqueued while pipelined host batches are in
    flight on the context's stream, waits for them (shared workspace), and a host batch
    submitted after it waits for the device batch: every result equals the batch run alone."""
    import torch
    pb = problems.build("refine_o1_ovs", n_particles=12, seed=14, diff2_mode=1)
    P = pb["parts"]
    es = pb["product"]()
    halves = [(0, 6), (6, 12)]

    def part(a, b):
        return P["fimg"][a:b], P["ctf"][a:b], P["minv"][a:b], P["scalars"][a:b]

    ref = [es.expectation(*part(a, b)) for a, b in halves]
    dev = torch.device("cuda")
    a, b = halves[1]
    n = b - a
    fimg = torch.from_numpy(np.ascontiguousarray(P["fimg"][a:b]).view(np.float32)).to(dev)
    ctf = torch.from_numpy(np.ascontiguousarray(P["ctf"][a:b])).to(dev)
    minv = torch.from_numpy(np.ascontiguousarray(P["minv"][a:b])).to(dev)
    scal = torch.from_numpy(np.ascontiguousarray(P["scalars"][a:b])).to(dev)
    host = es._result_arrays(n)
    tmap = {np.dtype("float64"): torch.float64, np.dtype("int64"): torch.int64, np.dtype("int32"): torch.int32}
    res = {k: torch.zeros(v.shape, dtype=tmap[v.dtype], device=dev) for k, v in host.items()}
    ptrs = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
    stream = torch.cuda.Stream()
    t0, got0 = es.expectation_submit(*part(*halves[0]))
    es.expectation_device(n, ctypes.c_void_p(fimg.data_ptr()), ctypes.c_void_p(ctf.data_ptr()),
                          ctypes.c_void_p(minv.data_ptr()), ctypes.c_void_p(scal.data_ptr()), ptrs,
                          stream=stream.cuda_stream)
    t2, got2 = es.expectation_submit(*part(*halves[0]))
    es.wait()
    stream.synchronize()
    got1 = {k: v.cpu().numpy() for k, v in res.items()}
    for got, r in ((got0, ref[0]), (got1, ref[1]), (got2, ref[0])):
        assert np.all(got["status"] == 0)
        assert np.array_equal(got["pose"], r["pose"])
        assert np.array_equal(got["nr_sign"], r["nr_sign"])
        assert np.allclose(got["sum_weight"], r["sum_weight"], rtol=1e-9, atol=0)
    es.close()


def test_autotune_waits_for_host_batches_in_flight():
    """Two pipelined host batches (one per staging slot, their results read back on a
    separate stream) are still in flight when t2b_autotune runs tuning batches on slot 0's
    buffers: the tuner waits for them, both keep their own results, and a batch submitted
    after the tuner (slot 0 again) gives the results of the same batch run alone."""
    pb = problems.build("refine_o1_ovs", n_particles=12, seed=15, diff2_mode=1)
    P = pb["parts"]
    es = pb["product"]()
    halves = [(0, 6), (6, 12)]

    def part(a, b):
        return P["fimg"][a:b], P["ctf"][a:b], P["minv"][a:b], P["scalars"][a:b]

    ref = [es.expectation(*part(a, b)) for a, b in halves]
    t0, got0 = es.expectation_submit(*part(*halves[0]))
    t1, got1 = es.expectation_submit(*part(*halves[1]))
    es.autotune(*part(0, 12))
    es.wait(t1)
    t2, got2 = es.expectation_submit(*part(*halves[0]))
    es.wait()
    for got, r in ((got0, ref[0]), (got1, ref[1]), (got2, ref[0])):
        assert np.all(got["status"] == 0)
        assert np.array_equal(got["pose"], r["pose"])
        assert np.array_equal(got["nr_sign"], r["nr_sign"])
        # the tuned tile shapes change no FP64 sum beyond rounding
        assert np.allclose(got["sum_weight"], r["sum_weight"], rtol=1e-7, atol=0)
        assert np.allclose(got["min_diff2"], r["min_diff2"], rtol=1e-7, atol=0)
    es.close()
