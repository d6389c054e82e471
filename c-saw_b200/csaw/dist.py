"""Multi-GPU placement: replicas, each with its own share of the samples.

Samples and walks are independent units, so the work shards with no data-path
collective (the reference's MPI launcher splits #samples the same way,
non-stream/mpi_main.cpp:38).  Every sample keeps its global id through
csaw_params.sample_base, so the Philox keys -- and therefore the edges -- do
not depend on how the job is split: the union of the shards equals the
single-GPU output.  The only collectives are the final count/time reductions.
"""
import ctypes

from . import _lib


def shard_range(n, rank, world):
    """Contiguous [lo, hi) share of n units for rank (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return n * rank // world, n * (rank + 1) // world


def _copy(p):
    q = _lib.Params()
    ctypes.pointer(q)[0] = p
    return q


def shard_params(p, rank, world):
    """Params of rank's shard of job p (strong scaling) and its seed slice."""
    lo, hi = shard_range(p.n_samples, rank, world)
    q = _copy(p)
    q.n_samples = hi - lo
    q.sample_base = p.sample_base + lo
    per = 1 if p.mode == _lib.MODE_WALK else p.frontier_size
    return q, slice(lo * per, hi * per)


def replica_params(p, rank):
    """Params of rank's replica for weak scaling: the same job shape on the
    next block of sample ids, so no two ranks produce the same sample."""
    q = _copy(p)
    q.sample_base = p.sample_base + rank * p.n_samples
    return q


def reduce_totals(edges, seconds, group=None):
    """(sum of edges, max of seconds) over the ranks of the default group."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(edges), float(seconds)], dtype=torch.float64, device=dev)
    e, s = t[0:1].clone(), t[1:2].clone()
    dist.all_reduce(e, group=group)
    dist.all_reduce(s, op=dist.ReduceOp.MAX, group=group)
    return float(e.item()), float(s.item())
