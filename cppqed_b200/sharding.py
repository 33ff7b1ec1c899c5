"""Trajectory sharding over ranks (one process per GPU).

MCWF trajectories are independent, so an ensemble of N trajectories per rank over W ranks
is W disjoint blocks of random streams: rank r runs streams
``prng_stream + r * N ... prng_stream + (r + 1) * N - 1``, exactly the trajectories
``r * N ...`` of one ensemble of W * N (the reference's Ensemble gives trajectory i the
stream prngStream + i, MCWF_Trajectory.h:223-226).  The only exchange is the sum of the
per-rank ensemble sums after every output interval (a few hundred bytes), and timings are
reduced to their maximum over ranks.  The helpers work with any torch.distributed backend
(NCCL with CUDA tensors, gloo with CPU tensors).
"""
import numpy as np


def first_stream(prng_stream, n_per_rank, rank):
    """First random stream of this rank's block of trajectories."""
    return int(prng_stream) + int(rank) * int(n_per_rank)


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def allreduce_sum(x, world):
    """Element-wise sum over ranks of a float64 array (identity for one rank)."""
    x = np.asarray(x, dtype=np.float64)
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor(x, dtype=torch.float64, device=_device())
    dist.all_reduce(t)
    return t.cpu().numpy()


def max_over_ranks(x, world):
    """Element-wise maximum over ranks (the timing rule: a step takes as long as the
    slowest rank)."""
    x = np.asarray(x, dtype=np.float64)
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor(x, dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().numpy()
