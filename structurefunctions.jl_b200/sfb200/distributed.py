"""Multi-GPU: one process per GPU, one all-reduce.

The pair set of one call is cut into the upper-triangle tile pairs of the kernels, which are
independent units of work. Every rank holds all points (they are small), runs one contiguous shard of
the tile pairs (sfb200_plan_set_option SFB200_OPT_SHARD; shards hold equal numbers of pairs, see
sfb200_shard_bounds) into a partial histogram, and a single all-reduce (NCCL over NVLink on GPUs, gloo
on CPUs) adds the partial sums (FP64) and counts (int64).
This mirrors the reference's MPI rank sharding (ext/StructureFunctionsMPIExt.jl:24-26, one reduction
of the per-rank histograms), with tile pairs in place of outer-loop indices.
"""
import numpy as np

from . import _abi, _lib
from .api import plan_description


def shard_value(index, count):
    """The SFB200_OPT_SHARD value of shard `index` of `count`."""
    if not 0 <= index < count:
        raise ValueError("shard index must be in [0, count)")
    return (int(count) << 32) | int(index)


def shard_bounds(n, tile, index, count):
    """Tile pairs [lo, hi) of shard `index` of `count` for n points in tiles of `tile` points: the
    library's partition (sfb200_shard_bounds, host arithmetic only), contiguous ranges of tile pairs
    each within one tile pair of an equal share of the pairs."""
    import ctypes as C

    lo, hi = C.c_int64(), C.c_int64()
    rc = _lib.load().sfb200_shard_bounds(int(n), int(tile), int(index), int(count), C.byref(lo), C.byref(hi))
    if rc != 0:
        raise ValueError("invalid shard request")
    return lo.value, hi.value


def tile_pair_pairs(n, tile, ti, tj):
    """Pairs of tile pair (ti, tj): s_i s_j off the diagonal, s (s - 1) / 2 on it."""
    si = min(tile, n - ti * tile)
    sj = min(tile, n - tj * tile)
    return si * (si - 1) // 2 if ti == tj else si * sj


def allreduce_histogram(sums, counts, group=None):
    """Add the partial histograms of all ranks in place (torch tensors on the backend's device)."""
    import torch.distributed as dist

    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    return sums, counts


def sharded_run(ctx, ops, x, u, distance_bins, value_bins=None, distance_metric=None, precision="mixed",
                group=None):
    """Run one call across the ranks of `group` (one GPU each, current CUDA device = the rank's GPU).

    Returns the full histogram on every rank as host arrays (sums float64, counts uint64).
    """
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    x = np.asfortranarray(x)
    u = np.asfortranarray(u)
    desc, keep = plan_description(ops, u.shape[0], distance_bins, value_bins, distance_metric, precision,
                                  x.dtype, u.dtype)
    plan = _lib.Plan(ctx, desc, keep)
    try:
        plan.set_option(_abi.OPT_SHARD, shard_value(rank, world))
        dev = torch.device("cuda", torch.cuda.current_device())
        sums = torch.zeros(plan.n_sums, dtype=torch.float64, device=dev)
        counts = torch.zeros(plan.n_counts, dtype=torch.int64, device=dev)
        plan.run(x.ctypes.data, u.ctypes.data, x.shape[1], _abi.RUN_DEVICE_OUTPUT, sums.data_ptr(),
                 counts.data_ptr(), ctx.stream)
        torch.cuda.synchronize()
        allreduce_histogram(sums, counts, group)
        return sums.cpu().numpy(), counts.cpu().numpy().astype(np.uint64)
    finally:
        plan.close()
