"""The grid exchange of t2relion_b200.parallel on the library's device grids through NCCL: one
rank (one GPU), so the all-reduce within its gold-standard half must leave the grids as they
are, and a write through the zero-copy DLPack view must land in the library's own grid.  The
same code runs over NVLink with more ranks; those are covered on CPU ranks (gloo) by
tests/test_parallel_gloo.py and tests/test_jobfarm.py."""
import os

import numpy as np
import pytest

import problems
from conftest import load_package
from test_parallel_gloo import _free_port

pytestmark = pytest.mark.gpu


def _child(rank, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="1",
                      NCCL_NVLS_ENABLE="0")
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    load_package()
    import t2relion_b200.parallel as par
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60))
    pb = problems.build("refine_o2", n_particles=16, seed=47, nr_classes=2)
    P = pb["parts"]
    es = pb["product"]()
    res = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    before = [es.get_backprojector(k) for k in range(2)]
    halves = par.gold_standard_groups(1)
    par.allreduce_grids_(es, 2, group=halves.mine)
    torch.cuda.synchronize()
    after = [es.get_backprojector(k) for k in range(2)]
    sums = par.reduce_wsums([res], group=halves.mine)
    # a write through the view of class 1's weights reaches the library's grid
    nvox = int(np.prod(es._grid_shape))
    _, w_ptr = es.backprojector_device_ptrs(1)
    view = par.device_view(w_ptr, nvox, 0)
    view.mul_(2.0)
    dist.all_reduce(view, group=halves.mine)
    torch.cuda.synchronize()
    doubled = es.get_backprojector(1)[1]
    del view
    np.savez(os.path.join(outdir, "exchange.npz"),
             d0=before[0][0], w0=before[0][1], d1=before[1][0], w1=before[1][1],
             a0=after[0][0], aw0=after[0][1], a1=after[1][0], aw1=after[1][1], doubled=doubled,
             sumw=sums["sumw"], sumw_ref=np.asarray(res["sumw"], np.float64).sum(axis=0), ranks=halves.ranks[0])
    es.close()
    dist.destroy_process_group()


def test_nccl_exchange_on_library_grids(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_child, args=(_free_port(), str(tmp_path)), nprocs=1, start_method="spawn", join=True)
    r = np.load(tmp_path / "exchange.npz")
    assert list(r["ranks"]) == [0]
    for a, b in (("d0", "a0"), ("w0", "aw0"), ("d1", "a1"), ("w1", "aw1")):
        assert np.array_equal(r[a], r[b]), a
    assert np.max(np.abs(r["w0"])) > 0 and np.max(np.abs(r["w1"])) > 0
    assert np.array_equal(r["doubled"], 2.0 * r["w1"])
    assert np.allclose(r["sumw"], r["sumw_ref"], rtol=1e-12)
