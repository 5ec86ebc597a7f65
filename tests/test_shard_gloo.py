"""Multi-GPU host logic on CPU: two gloo ranks shard one search into disjoint
offset ranges, re-derive each other's keys, and reduce timings by maximum."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from onion_gen_b200 import key, shard, workloads

        seed = workloads.seed(42)
        start = shard.rank_start(seed, rank)
        # the rank's 5th candidate, offset 8*5 locally, is the search's global offset
        local = 40
        g = shard.global_offset(rank, local)
        sec = O.expanded_secret_at_offset(seed, g)
        want = O.pack(O.scalar_base_mult(sec[:32]))
        got = O.chain_keys(start, 8, 8, signed=True)[32 * 5: 32 * 6]
        ok = want == got
        packed = bytearray(got)
        packed[31] &= 0x7F
        key.check_hit(seed, g, bytes(packed))
        mx = shard.max_over_ranks([1.0 + rank, 10.0 - rank])
        scalars = [None] * world
        dist.all_gather_object(scalars, int.from_bytes(shard.rank_scalar(seed, rank), "little"))
        q.put((rank, ok, mx, scalars))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_disjoint_ranges():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from onion_gen_b200 import shard

    for rank, ok, mx, scalars in out:
        assert ok, rank
        assert mx == [2.0, 10.0]
        assert scalars[1] - scalars[0] == 1 << shard.RANK_SHIFT


def _lease_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from onion_gen_b200 import key, shard

        mine = shard.lease_blocks(1000, 11, rank, world)
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        seeds = [key.block_seed(bytes(range(32)), b).hex() for b in mine]
        all_seeds = [None] * world
        dist.all_gather_object(all_seeds, seeds)
        q.put((rank, shares, all_seeds))
    finally:
        dist.destroy_process_group()


def test_three_gloo_ranks_split_a_lease():
    """A leased range of 11 blocks over three ranks: every block exactly once,
    each searched from its own block seed, whatever rank takes it."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_lease_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from onion_gen_b200 import key, shard

    for rank, shares, all_seeds in out:
        flat = sorted(b for s in shares for b in s)
        assert flat == list(range(1000, 1011))
        assert shares[rank] == shard.lease_blocks(1000, 11, rank, 3)
        seeds = [s for ss in all_seeds for s in ss]
        assert len(set(seeds)) == 11
        assert sorted(seeds) == sorted(key.block_seed(bytes(range(32)), b).hex() for b in range(1000, 1011))
    import pytest as _pytest

    with _pytest.raises(ValueError):
        shard.lease_blocks(0, 4, 2, 2)
