"""The leaderless job farm of t2relion_b200.parallel against the reference's leader job loop
(oracle/jobfarm_oracle.py), and on gloo ranks: every particle is processed once, by a rank of
its own random subset, and the results equal one process's."""
import heapq
import os
import time

import numpy as np
import pytest

import jobfarm_oracle as jo
import problems
from conftest import load_package
from test_parallel_gloo import _free_port


def _par():
    load_package()
    import t2relion_b200.parallel as par
    return par


@pytest.mark.parametrize("n,followers,pool,guided", [(0, 2, 1, True), (1, 2, 5, True), (1000, 4, 8, True),
                                                     (1000, 1, 8, True), (999, 3, 7, False), (17, 8, 100, True)])
def test_farm_jobs_cover_the_range_in_order(n, followers, pool, guided):
    par = _par()
    jobs = par.farm_jobs(5, 5 + n - 1, followers, pool, guided)
    assert sum(b - a + 1 for a, b in jobs) == n
    assert all(b >= a for a, b in jobs)
    assert all(j1[1] + 1 == j2[0] for j1, j2 in zip(jobs, jobs[1:]))
    if n:
        assert jobs[0][0] == 5 and jobs[-1][1] == 5 + n - 1
    sizes = [b - a + 1 for a, b in jobs]
    if not guided:
        assert all(s == pool for s in sizes[:-1])
    elif followers == 1:
        assert len(jobs) == (1 if n else 0)
    else:
        assert all(s >= pool for s in sizes[:-1])
        assert sizes[:-1] == sorted(sizes[:-1], reverse=True)


def _simulate(grant, followers, speeds, seed):
    """Followers ask for a job, work on it for (particles x their speed + jitter) and ask again;
    requests are served in the order of the times they arrive.  grant(f) -> (first, last) or None.
    Returns the grants in order: (follower, first, last)."""
    rng = np.random.default_rng(seed)
    queue = [(rng.uniform(0, 1e-3), f) for f in range(1, followers + 1)]
    heapq.heapify(queue)
    out = []
    while queue:
        t, f = heapq.heappop(queue)
        job = grant(f)
        if job is None:
            continue
        out.append((f,) + tuple(job))
        heapq.heappush(queue, (t + (job[1] - job[0] + 1) * speeds[f - 1] + rng.uniform(0, 1e-3), f))
    return out


CASES = [(50, 101, 2, 4, True), (500, 1000, 4, 8, True), (500, 1000, 6, 3, True), (37, 78, 8, 2, True),
         (0, 10, 2, 1, True), (60, 60, 4, 5, True), (250, 500, 3, 10, True), (0, 1000, 3, 7, False),
         (0, 5, 4, 2, False)]


@pytest.mark.parametrize("n1,n,followers,pool,split", CASES)
def test_farm_grants_equal_the_leaders(n1, n, followers, pool, split):
    """The same request order gives the same ranges: the leader's loop restated, against one
    JobFarm per rank sharing a key-value store (rank r = follower r + 1)."""
    import torch.distributed as dist
    par = _par()
    speeds = np.random.default_rng(n + followers).uniform(0.5, 3.0, followers)
    leader = jo.Leader(n1, n, followers, pool, split)
    ref = _simulate(leader.request, followers, speeds, 1)
    store = dist.HashStore()
    farms = [par.JobFarm(store, n, pool, r, followers, split_halves=split, n_half1=n1, tag="t") for r in
             range(followers)]

    def grant(f):
        job = farms[f - 1].next_job()
        return None if job is None else job[1:]
    got = _simulate(grant, followers, speeds, 1)
    assert got == ref
    covered = sorted(p for _, a, b in got for p in range(a, b + 1))
    assert covered == list(range(n))
    if split:
        for f, a, b in got:
            assert (b < n1) == (f % 2 == 1), (f, a, b)


def test_single_rank_takes_both_subsets_and_tags_restart():
    import torch.distributed as dist
    par = _par()
    store = dist.HashStore()
    for tag in (0, 1):
        jobs = list(par.JobFarm(store, 30, 4, 0, 1, n_half1=12, tag=tag))
        assert jobs == [(1, 0, 11), (2, 12, 29)]
    with pytest.raises(ValueError):
        par.JobFarm(store, 30, 4, 2, 2)
    with pytest.raises(ValueError):
        par.JobFarm(store, 30, 4, 0, 2, n_half1=31)


def test_gather_jobs_checks_cover():
    par = _par()
    rows = np.arange(10)[:, None] * np.ones((1, 3))
    local = [(0, 3, rows[0:4]), (4, 9, rows[4:10])]
    assert np.array_equal(par.gather_jobs(local, 10), rows)
    with pytest.raises(ValueError):
        par.gather_jobs(local[:1], 10)
    with pytest.raises(ValueError):
        par.gather_jobs(local + [(2, 2, rows[2:3])], 10)


def _farm_worker(rank, world, port, outdir):
    """One rank: draws jobs of its random subset from the farm on the process group's store, runs
    the E-step on each (the FP64 oracle standing in for the GPU), then gathers the poses of all
    jobs and sums its half's grids and weighted sums."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    load_package()
    import t2relion_b200.parallel as par
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    store = dist.distributed_c10d._get_default_store()
    halves = par.gold_standard_groups(world)
    pb = problems.build("refine_o1_ovs", n_particles=16, seed=19)
    P = pb["parts"]
    mres = pb["sy"].mresol(pb["s"])
    farm = par.JobFarm(store, 16, 1, rank, world, split_halves=True, n_half1=8, tag="it1")
    local, results, mine = [], [], []
    rng = np.random.default_rng(rank)
    for subset, a, b in farm:
        assert subset == par.half_of(rank)
        op = pb["prob"].particles(P["fimg"][a:b + 1], P["ctf"][a:b + 1], P["minv"][a:b + 1], P["scalars"][a:b + 1], mres)
        res = pb["prob"].estep(op, nthreads=1)
        results.append(res)
        local.append((a, b, np.asarray(res["pose"])))
        mine.append((a, b))
        time.sleep(rng.uniform(0, 0.05))
    poses = par.gather_jobs(local, 16)
    data, weight = pb["prob"].grids()
    f64 = torch.from_numpy(np.ascontiguousarray(np.stack([data.real, data.imag], -1)))
    w64 = torch.from_numpy(np.ascontiguousarray(weight))
    dist.all_reduce(f64, op=dist.ReduceOp.SUM, group=halves.mine)
    dist.all_reduce(w64, op=dist.ReduceOp.SUM, group=halves.mine)
    sums = par.reduce_wsums(results, group=halves.mine)
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), poses=poses, jobs=np.array(mine).reshape(-1, 2),
             d64=f64.numpy(), w64=w64.numpy(), **sums)
    dist.barrier()
    dist.destroy_process_group()


def test_four_rank_farm_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    par = _par()
    mp.start_processes(_farm_worker, args=(4, _free_port(), str(tmp_path)), nprocs=4, start_method="spawn",
                       join=True)
    pb = problems.build("refine_o1_ovs", n_particles=16, seed=19)
    P = pb["parts"]
    full = pb["oracle_problem"]().estep(pb["oparts"], nthreads=2)
    red = [np.load(tmp_path / f"rank{r}.npz") for r in range(4)]
    granted = sorted(tuple(j) for r in red for j in r["jobs"])
    per_half = {1: par.farm_jobs(0, 7, 2, 1, True), 2: par.farm_jobs(8, 15, 2, 1, True)}
    assert granted == sorted(per_half[1] + per_half[2])
    for r in range(4):
        assert np.array_equal(red[r]["poses"], np.asarray(full["pose"]))
        for a, b in red[r]["jobs"]:
            assert (b <= 7) == (par.half_of(r) == 1)
    for h, idx in ((1, np.arange(0, 8)), (2, np.arange(8, 16))):
        r = [q for q in range(4) if par.half_of(q) == h][0]
        prob = pb["oracle_problem"]()
        op = prob.particles(P["fimg"][idx], P["ctf"][idx], P["minv"][idx], P["scalars"][idx], pb["sy"].mresol(pb["s"]))
        ref = prob.estep(op, nthreads=2)
        rd, rw = prob.grids()
        d64 = red[r]["d64"][..., 0] + 1j * red[r]["d64"][..., 1]
        assert np.allclose(d64, rd, rtol=1e-10, atol=1e-12) and np.allclose(red[r]["w64"], rw, rtol=1e-10, atol=1e-12)
        tot = par.reduce_wsums([ref])
        for k in par.SUMMED:
            assert np.allclose(red[r][k], tot[k], rtol=1e-10, atol=1e-300), k
