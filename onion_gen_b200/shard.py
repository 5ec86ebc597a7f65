"""Sharding one search across GPUs: independent offset ranges, no exchange.

Rank r of a world searches from base scalar s + r * 2^RANK_SHIFT, so its
offsets o (below 2^RANK_SHIFT) are the search's offsets r * 2^RANK_SHIFT + o:
ranges never meet and nothing crosses between GPUs but the final timing
reduction (onion-gen shards the same way, by independent blocks,
src/run.rs:1040-1049).
"""
from __future__ import annotations

from . import key

RANK_SHIFT = 43  # 2^43 / 8 = 2^40 candidates per rank before ranges could meet


def rank_scalar(seed: bytes, rank: int) -> bytes:
    s = int.from_bytes(key.secret_scalar(seed), "little") + (rank << RANK_SHIFT)
    return (s % (1 << 256)).to_bytes(32, "little")


def rank_start(seed: bytes, rank: int) -> bytes:
    """The start point of rank `rank`: (s + rank 2^RANK_SHIFT) B."""
    return key.scalar_base_mult(rank_scalar(seed, rank))


def global_offset(rank: int, offset: int) -> int:
    """A rank's local offset as an offset from the search's own scalar."""
    return (rank << RANK_SHIFT) + offset


def lease_blocks(first_block: int, blocks: int, rank: int, world: int):
    """The blocks of a leased range one rank searches: every world-th block,
    starting at first_block + rank. Each block is searched from its own seed
    (block_seed), as the reference's device workers each take blocks of the
    lease (src/run.rs:1040-1049); the ranks' shares are disjoint and cover
    the range."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(range(first_block + rank, first_block + blocks, world))


def max_over_ranks(values, group=None):
    """Element-wise maximum of per-rank timings (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.cpu().tolist()
