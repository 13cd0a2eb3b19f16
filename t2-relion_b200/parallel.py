"""Data-parallel E-step over several GPUs: one process per GPU.

Particles of an iteration are independent (the reference farms them out to MPI
followers, src/ml_optimiser_mpi.cpp:1155-1444), so every rank runs the E-step on
its own particles with no communication on the data path: a fixed shard
(`shard_range`) or jobs drawn from a shared counter (`JobFarm`, the leader's
job loop without a leader).  The one exchange is at
the end of the iteration: summing the backprojection grids and the weighted
sums over the ranks of one gold-standard half, which the reference does by a
device-to-host copy, a host double sum and MPI Send/Recv
(src/ml_optimiser_mpi.cpp:1465-1480, 1732-1830).  Here it is an in-place
all-reduce on the device grids through torch.distributed (NCCL over
NVLink/NVSwitch on GPUs, gloo on CPU).
"""
import ctypes

import numpy as np


def shard_range(n, rank, world):
    """Contiguous, balanced [begin, end) of `n` particles for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


# --- zero-copy torch view of library device memory (DLPack) -----------------
class _DLDevice(ctypes.Structure):
    _fields_ = [("device_type", ctypes.c_int32), ("device_id", ctypes.c_int32)]


class _DLDataType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class _DLTensor(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("device", _DLDevice), ("ndim", ctypes.c_int32),
                ("dtype", _DLDataType), ("shape", ctypes.POINTER(ctypes.c_int64)),
                ("strides", ctypes.POINTER(ctypes.c_int64)), ("byte_offset", ctypes.c_uint64)]


class _DLManagedTensor(ctypes.Structure):
    pass


_DELETER = ctypes.CFUNCTYPE(None, ctypes.POINTER(_DLManagedTensor))
_DLManagedTensor._fields_ = [("dl_tensor", _DLTensor), ("manager_ctx", ctypes.c_void_p),
                             ("deleter", _DELETER)]
_KEEP = {}


@_DELETER
def _release(ptr):
    _KEEP.pop(ctypes.addressof(ptr.contents), None)


def device_view(ptr, n_floats, device):
    """A float32 torch tensor aliasing `n_floats` floats at `ptr`: CUDA memory of device
    `device` (an int), or host memory when `device` is "cpu".

    The memory stays owned by whoever allocated it; the view must not outlive it.
    """
    import torch
    shape = (ctypes.c_int64 * 1)(n_floats)
    mt = _DLManagedTensor()
    mt.dl_tensor.data = ptr
    mt.dl_tensor.device = _DLDevice(1, 0) if device == "cpu" else _DLDevice(2, device)  # kDLCPU / kDLCUDA
    mt.dl_tensor.ndim = 1
    mt.dl_tensor.dtype = _DLDataType(2, 32, 1)  # kDLFloat, 32 bits
    mt.dl_tensor.shape = shape
    mt.dl_tensor.strides = None
    mt.dl_tensor.byte_offset = 0
    mt.manager_ctx = None
    mt.deleter = _release
    _KEEP[ctypes.addressof(mt)] = (mt, shape)
    pycapsule_new = ctypes.pythonapi.PyCapsule_New
    pycapsule_new.restype = ctypes.py_object
    pycapsule_new.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    cap = pycapsule_new(ctypes.addressof(mt), b"dltensor", None)
    return torch.utils.dlpack.from_dlpack(cap)


def allreduce_grids_(grids, nr_classes, group=None):
    """Sum the BP grids of every class over the ranks of `group`, in place (FP32, as the
    device grids hold them).

    `grids`: a t2relion_b200.EStep (the library's device grids, t2b_backprojector_device_ptrs;
    NCCL over NVLink) or any object with the same backprojector_device_ptrs(k) and _grid_shape
    whose `device` attribute is "cpu" (host grids; gloo).  The views alias the memory: no
    copy, the reduction writes the grids themselves.
    """
    import torch
    import torch.distributed as dist
    dev = getattr(grids, "device", None)
    if dev != "cpu":
        dev = torch.cuda.current_device()
    nvox = int(np.prod(grids._grid_shape))
    for k in range(nr_classes):
        data_ptr, w_ptr = grids.backprojector_device_ptrs(k)
        for ptr, n in ((data_ptr, 2 * nvox), (w_ptr, nvox)):
            dist.all_reduce(device_view(ptr, n, dev), op=dist.ReduceOp.SUM, group=group)


class Halves:
    """The two gold-standard halves of one job as process groups."""

    def __init__(self, groups, ranks, rank):
        self.groups, self.ranks = groups, ranks
        self.index = 0 if rank in ranks[0] else 1     # 0: random subset 1, 1: random subset 2
        self.mine = groups[self.index]
        self.sizes = [len(r) for r in ranks]


def half_of(rank):
    """Random subset (1 or 2) of torch rank `rank`.  Rank r plays the reference's follower r + 1;
    followers of odd MPI rank form subset 1, even ones subset 2 (MpiNode::myRandomSubset,
    src/mpi.cpp:90-96), and each subset's weighted sums and grids are summed over its own
    followers only (combineAllWeightedSums, src/ml_optimiser_mpi.cpp:1732-1830)."""
    return 1 if rank % 2 == 0 else 2


def gold_standard_groups(world, rank=None):
    """Process groups of the two halves (every rank creates both: dist.new_group is collective).
    A world of one rank has one group holding both halves' data (no exchange is needed)."""
    import torch.distributed as dist
    rank = dist.get_rank() if rank is None else rank
    ranks = [[r for r in range(world) if half_of(r) == h] for h in (1, 2)]
    groups = [dist.new_group(r) if r else None for r in ranks]
    return Halves(groups, ranks, rank)


class HostGrids:
    """Backprojection grids in host memory with the EStep grid interface (float32 data
    interleaved re/im and weight, [K] x grid), for the exchange on CPU ranks (gloo)."""
    device = "cpu"

    def __init__(self, data, weight):
        w = np.asarray(weight)
        self._grid_shape = w.shape[1:]
        self.data = np.ascontiguousarray(np.stack([np.asarray(data).real, np.asarray(data).imag], -1), np.float32)
        self.weight = np.ascontiguousarray(w, np.float32)

    def backprojector_device_ptrs(self, k):
        return self.data[k].ctypes.data, self.weight[k].ctypes.data

    def grids(self):
        return self.data[..., 0] + 1j * self.data[..., 1], self.weight


# --- particle jobs: the leader's job loop without a leader --------------------
def farm_jobs(first, last, followers, nr_pool, guided):
    """The particle jobs [(first, last), ...] the reference's leader hands out, in the order it
    grants them, for the particles first..last (inclusive) of one random subset
    (MlOptimiserMpi::expectation, src/ml_optimiser_mpi.cpp:1187-1227).  With `guided` (split
    random halves) and more than one follower per half, each job is the particles still to do
    over 2 x followers, rounded up, at least nr_pool; with one follower the whole subset is one
    job.  Otherwise (no split halves) jobs are nr_pool particles.  The k-th grant's range depends
    on k alone, so any rank that draws ticket k can compute it."""
    todo = last - first + 1
    if todo <= 0:
        return []
    if nr_pool < 1 or followers < 1:
        raise ValueError("nr_pool and followers must be >= 1")
    jobs, done = [], 0
    while done < todo:
        if not guided:
            n = nr_pool
        elif followers == 1:
            n = todo
        else:
            n = max(nr_pool, (todo - done + 2 * followers - 1) // (2 * followers))
        n = min(n, todo - done)
        jobs.append((first + done, first + done + n - 1))
        done += n
    return jobs


class JobFarm:
    """Dynamic distribution of an iteration's particles over the ranks, in place of the
    leader/follower exchange of the reference (src/ml_optimiser_mpi.cpp:1155-1444: followers
    send a job request, the leader replies with the next particle range and the images, the
    follower runs expectationSomeParticles on it and sends the metadata back).

    Here there is no leader rank: every rank reads its particles itself (the reference's
    parallel disc I/O) and draws the next job of its random subset with one atomic add on the
    torch.distributed key-value store (a ticket; the k-th ticket is the k-th job of
    `farm_jobs`).  A rank that finishes early draws again, so slow and fast GPUs balance as they
    do under the leader.  With split random halves (gold-standard refinement) rank r plays
    follower r + 1: even ranks take the particles of subset 1 (0 .. n_half1 - 1), odd ranks those
    of subset 2, and each subset counts world // 2 followers ((size - 1) / 2 in the reference);
    a single rank takes both subsets in turn.  Keys are scoped by `tag` (e.g. the iteration), so
    each iteration starts from ticket 0 without resetting the store."""

    def __init__(self, store, n_particles, nr_pool, rank, world, split_halves=True, n_half1=None, tag=0):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank / world")
        self.store, self.rank, self.world, self.tag = store, rank, world, tag
        if split_halves:
            n1 = (n_particles + 1) // 2 if n_half1 is None else n_half1
            if not 0 <= n1 <= n_particles:
                raise ValueError("n_half1 out of range")
            per_half = max(1, world // 2)
            subsets = {1: farm_jobs(0, n1 - 1, per_half, nr_pool, True),
                       2: farm_jobs(n1, n_particles - 1, per_half, nr_pool, True)}
            self.order = [1, 2] if world == 1 else [half_of(rank)]
        else:
            subsets = {0: farm_jobs(0, n_particles - 1, world, nr_pool, False)}
            self.order = [0]
        self.subsets = subsets

    def _key(self, subset):
        return f"t2b_jobfarm/{self.tag}/{subset}"

    def next_job(self):
        """(subset, first, last) of the next job for this rank, or None when its subsets are done."""
        while self.order:
            subset = self.order[0]
            ticket = int(self.store.add(self._key(subset), 1)) - 1
            jobs = self.subsets[subset]
            if ticket < len(jobs):
                return (subset,) + jobs[ticket]
            self.order.pop(0)
        return None

    def __iter__(self):
        while True:
            job = self.next_job()
            if job is None:
                return
            yield job


def gather_jobs(local, n_particles, group=None):
    """Collect every rank's per-job results into particle order, as the leader's
    setMetaDataSubset does with the metadata the followers send back
    (src/ml_optimiser_mpi.cpp:1166-1180).  `local`: list of (first, last, rows) with rows an
    array of last - first + 1 rows.  Returns the (n_particles, ...) array on every rank; raises
    if the jobs do not cover each particle exactly once."""
    import torch.distributed as dist
    parts = [local]
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, local, group=group)
    seen = np.zeros(n_particles, np.int64)
    out = None
    for first, last, rows in (j for p in parts for j in p):
        rows = np.asarray(rows)
        if rows.shape[0] != last - first + 1 or first < 0 or last >= n_particles:
            raise ValueError(f"job {first}..{last}: {rows.shape[0]} rows")
        if out is None:
            out = np.zeros((n_particles,) + rows.shape[1:], rows.dtype)
        out[first:last + 1] = rows
        seen[first:last + 1] += 1
    if n_particles and not np.all(seen == 1):
        raise ValueError(f"particles not covered exactly once: {np.flatnonzero(seen != 1)[:8]}")
    return out


# per-particle fields of a result dict that are summed into the model
SUMMED = ("wsum_sigma2", "wsum_pdf_class", "wsum_pdf_dir", "wsum_norm", "sumw", "wsum_sigma2_offset")


def reduce_wsums(results, group=None):
    """Sum the weighted sums of this rank's particles, then over the ranks (FP64).

    `results`: list of result dicts of t2relion_b200.EStep.expectation.  Returns a
    dict of summed arrays, identical on every rank of `group`.
    """
    import torch
    import torch.distributed as dist
    out = {}
    for key in SUMMED:
        local = sum(np.asarray(r[key], np.float64).sum(axis=0) for r in results)
        t = torch.as_tensor(np.atleast_1d(local), dtype=torch.float64)
        if dist.is_initialized() and dist.get_world_size(group) > 1:
            if dist.get_backend(group) == "nccl":
                t = t.cuda()
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[key] = t.cpu().numpy()
    return out
