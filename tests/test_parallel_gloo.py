"""Multi-rank logic of the data-parallel E-step on CPU (gloo, world size 2).

Each rank takes its particle shard, runs the E-step on it (the FP64 oracle
stands in for the GPU here), and the reductions of t2relion_b200.parallel must
reproduce the totals of one process over all particles: the weighted sums and
the backprojection grids (which are linear in the particles).
"""
import os
import socket
import sys

import numpy as np
import pytest

import problems
from conftest import load_package


def test_shard_range_partitions():
    load_package()
    import t2relion_b200.parallel as par
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            spans = [par.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - s for s, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        par.shard_range(10, 2, 2)


def _worker(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    load_package()
    import t2relion_b200.parallel as par
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    pb = problems.build("refine_o1_ovs", n_particles=10, seed=17)
    b0, b1 = par.shard_range(10, rank, world)
    P = pb["parts"]
    op = pb["prob"].particles(P["fimg"][b0:b1], P["ctf"][b0:b1], P["minv"][b0:b1], P["scalars"][b0:b1],
                              pb["sy"].mresol(pb["s"]))
    res = pb["prob"].estep(op, nthreads=2)
    sums = par.reduce_wsums([res])
    data, weight = pb["prob"].grids()
    t = torch.from_numpy(np.ascontiguousarray(np.stack([data.real, data.imag], -1)))
    tw = torch.from_numpy(np.ascontiguousarray(weight))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    dist.all_reduce(tw, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.savez(os.path.join(outdir, "reduced.npz"), data=t.numpy(), weight=tw.numpy(),
                 **{k: v for k, v in sums.items()})
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_reduction_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    load_package()
    import t2relion_b200.parallel as par
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    red = np.load(tmp_path / "reduced.npz")
    pb = problems.build("refine_o1_ovs", n_particles=10, seed=17)
    full = pb["prob"].estep(pb["oparts"], nthreads=2)
    data, weight = pb["prob"].grids()
    ref = par.reduce_wsums([full])
    for k in par.SUMMED:
        assert np.allclose(red[k], ref[k], rtol=1e-12, atol=1e-300), k
    assert np.allclose(red["data"][..., 0] + 1j * red["data"][..., 1], data, rtol=1e-10, atol=1e-12)
    assert np.allclose(red["weight"], weight, rtol=1e-10, atol=1e-12)


def _halves_worker(rank, world, port, outdir):
    """One rank of a 4-rank job: its shard's E-step (FP64 oracle standing in for the GPU), its
    grids as FP32 host grids, and the exchange of the library's parallel module within its
    gold-standard half: allreduce_grids_ on the FP32 grids through the same DLPack views the
    device grids use, and an FP64 all-reduce of the same grids as the reference's host sum."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    load_package()
    import t2relion_b200.parallel as par
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    halves = par.gold_standard_groups(world)
    pb = problems.build("refine_o1_ovs", n_particles=16, seed=19)
    b0, b1 = par.shard_range(16, rank, world)
    P = pb["parts"]
    op = pb["prob"].particles(P["fimg"][b0:b1], P["ctf"][b0:b1], P["minv"][b0:b1], P["scalars"][b0:b1],
                              pb["sy"].mresol(pb["s"]))
    res = pb["prob"].estep(op, nthreads=1)
    data, weight = pb["prob"].grids()
    hg = par.HostGrids(data, weight)
    par.allreduce_grids_(hg, 1, group=halves.mine)
    f64 = torch.from_numpy(np.ascontiguousarray(np.stack([data.real, data.imag], -1)))
    w64 = torch.from_numpy(np.ascontiguousarray(weight))
    dist.all_reduce(f64, op=dist.ReduceOp.SUM, group=halves.mine)
    dist.all_reduce(w64, op=dist.ReduceOp.SUM, group=halves.mine)
    sums = par.reduce_wsums([res], group=halves.mine)
    if rank in (0, 1):   # the first rank of each half writes that half's totals
        d32, w32 = hg.grids()
        np.savez(os.path.join(outdir, f"half{par.half_of(rank)}.npz"), d32=d32, w32=w32,
                 d64=f64.numpy(), w64=w64.numpy(), ranks=np.array(halves.ranks[halves.index]), **sums)
    dist.barrier()
    dist.destroy_process_group()


def test_gold_standard_halves_exchange(tmp_path):
    """4 ranks: halves {0, 2} and {1, 3} (the reference's followers 1, 3 and 2, 4).  Each half's
    FP32 grid sum through allreduce_grids_ matches the FP64 sum of the same grids (FSC >= 0.999
    per shell, max error 1e-6 of the largest voxel) and a single process over that half's
    particles (FP64 sums to 1e-10); the two halves stay different."""
    import torch.multiprocessing as mp
    load_package()
    import t2relion_b200.parallel as par
    assert [par.half_of(r) for r in range(4)] == [1, 2, 1, 2]
    mp.start_processes(_halves_worker, args=(4, _free_port(), str(tmp_path)), nprocs=4, start_method="spawn",
                       join=True)
    pb = problems.build("refine_o1_ovs", n_particles=16, seed=19)
    P = pb["parts"]
    shells = problems.shells_of(pb["prob"].gshape[1:])
    nsh = 2 * pb["r"] + 1
    out = {}
    for h in (1, 2):
        red = np.load(tmp_path / f"half{h}.npz")
        assert list(red["ranks"]) == [r for r in range(4) if par.half_of(r) == h]
        d64 = red["d64"][..., 0] + 1j * red["d64"][..., 1]
        d32 = red["d32"][0]
        f = problems.fsc(d32.reshape(-1), d64[0].reshape(-1), shells, shells.max() + 1)
        assert np.all(f[1:nsh] >= 0.999), f[:nsh]
        assert np.max(np.abs(d32 - d64[0])) <= 1e-6 * np.max(np.abs(d64[0]))
        assert np.max(np.abs(red["w32"][0] - red["w64"][0])) <= 1e-6 * np.max(red["w64"][0])
        # a single process over the half's particles
        idx = np.concatenate([np.arange(*par.shard_range(16, r, 4)) for r in red["ranks"]])
        prob = pb["oracle_problem"]()
        op = prob.particles(P["fimg"][idx], P["ctf"][idx], P["minv"][idx], P["scalars"][idx], pb["sy"].mresol(pb["s"]))
        ref = prob.estep(op, nthreads=2)
        rd, rw = prob.grids()
        assert np.allclose(d64, rd, rtol=1e-10, atol=1e-12) and np.allclose(red["w64"], rw, rtol=1e-10, atol=1e-12)
        tot = par.reduce_wsums([ref])
        for k in par.SUMMED:
            assert np.allclose(red[k], tot[k], rtol=1e-10, atol=1e-300), k
        out[h] = d64
    assert np.max(np.abs(out[1] - out[2])) > 0.1 * np.max(np.abs(out[1]))
