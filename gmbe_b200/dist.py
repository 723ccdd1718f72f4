"""Several GPUs of one node, one process each (torch.distributed).

Root subtrees are independent and the count and set hash are sums mod 2^64,
so N ranks enumerate interleaved shares of the degree-ordered roots (rank r
takes positions p = r mod N, counted from the top, which balances the heavy
roots) and one all-reduce of two int64 combines them.  The reference has
multi-GPU root stealing through managed memory (src/IterFinderGpu.cu:1250-1288);
no data-path collective is needed here.
"""
from __future__ import annotations

MASK64 = (1 << 64) - 1


def shard_params(rank: int, world: int) -> dict:
    """mbe_params fields that select this rank's share of the roots."""
    return dict(shard_count=world, shard_index=rank) if world > 1 else {}


def _to_i64(x: int) -> int:
    x &= MASK64
    return x - (1 << 64) if x >= 1 << 63 else x


def sum_results(count: int, set_hash: int, device=None, group=None) -> tuple[int, int]:
    """Sums (count, set_hash) over the ranks, mod 2^64 (a no-op without a
    process group).  The two words travel as int64; two's-complement addition
    is addition mod 2^64."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([_to_i64(count), _to_i64(set_hash)], dtype=torch.int64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
    c, h = t.tolist()
    return c & MASK64, h & MASK64
