"""Multi-GPU plumbing for one COUNT query split across ranks.

Every rank holds the whole trie (0.3-1.3 GB at the benchmark sizes; HBM is
180 GB) and runs the work items i with i % world == rank of the shared,
heaviest-first plan (eh_exec_config.shard_index / shard_count).  The only
exchange is the final sum: one 8-byte all-reduce.  Counts are modulo 2^64
like the reference's signed long, so the sum is taken on int64 tensors and
read back as uint64 bit patterns.  The reference's own parallelism is the
same split over threads (par::for_range + par::reducer,
storage_engine/src/utils/parallel.cpp:42-79, utils/parallel.hpp:8-34).
"""
import torch

MASK64 = (1 << 64) - 1


def to_i64(u):
    """uint64 bit pattern -> int64 value with the same bits."""
    u &= MASK64
    return u - (1 << 64) if u >= (1 << 63) else u


def combine_counts(count, device="cpu", group=None):
    """Sum of every rank's partial count, modulo 2^64."""
    import torch.distributed as dist
    t = torch.tensor([to_i64(int(count))], dtype=torch.int64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
    return int(t.item()) & MASK64


def max_over_ranks(x, device="cpu", group=None):
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def owned(n_items, rank, world):
    """Indices of the work items a rank runs (host mirror of the device rule)."""
    return range(rank, n_items, world)
