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
