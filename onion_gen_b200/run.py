"""The device search loop of onion-gen's run driver (src/run.rs:1030-1119).

``device_search`` drives one ``gpu.Engine`` the way ``run::device_worker``
does: advance, confirm every survivor exactly against the filter set (on the
device for suffixes, whose address needs the sign bit and checksum), re-derive
the key of every match from its offset on the host and compare it with the
device's bytes, and stop once ``quota`` hits are in hand. It returns the
first ``quota`` hits in offset order: every advance covers the next contiguous
range of offsets, so once the quota is reached nothing below the last examined
offset is missing.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import filter as F
from . import gpu, key


@dataclass(frozen=True)
class Found:
    offset: int
    packed: bytes
    public_key: bytes
    filter: int


def device_search(device, seed: bytes, prefixes, quota: int, threads: int = 0, config=None, max_advances=None,
                  device_match=False):
    """``device_match`` moves the exact match onto the device
    (og_engine_advance_matches): only matches cross back, the same ones the
    host match finds."""
    fs = F.FilterSet.parse_all(prefixes)
    start = key.start_point(seed)
    np_ = fs.prefix_count()
    if np_ < len(fs):
        # suffixes: the filter engine (both bitmaps, the device match on)
        eng = gpu.Engine(device, start, filters=fs, config=config)
        device_match = True
    else:
        words, bits = fs.index_words()
        eng = gpu.Engine(device, start, threads=threads, bitmap=words, bitmap_bits=bits, config=config)
        if device_match:
            eng.match_on_device(fs)
    texts = fs.texts()
    found = []
    advances = 0
    examined = 0
    launch = eng.launch_matches if device_match else eng.launch
    launched = 0
    per_advance = eng.batch() * fs.match_probability()  # expected hits of one advance
    try:
        while len(found) < quota:
            if max_advances is not None and advances >= max_advances:
                break
            # keep the next advance running while this one is checked, unless
            # one advance is expected to bring four times the hits still
            # needed: then the second would almost surely go unused
            depth = 1 if per_advance >= 4 * (quota - len(found)) else 2
            while launched - advances < depth and (max_advances is None or launched < max_advances):
                launch()
                launched += 1
            if device_match:
                offsets, packed, matched = eng.collect_matches_raw()
                idx = np.arange(len(offsets))
            else:
                offsets, packed = eng.collect_raw()
                matched = fs.match_many(packed)  # the bitmap says maybe, the exact check decides
                idx = np.nonzero(matched >= 0)[0]
            advances += 1
            examined += eng.batch()
            # this advance's range lies above every earlier one: its matches
            # in offset order are the next hits, up to the quota
            for j in idx[np.argsort(offsets[idx], kind="stable")]:
                off, b, f = int(offsets[j]), bytes(packed[j]), int(matched[j])
                pk, _ = key.check_hit(seed, off, b)
                # confirmed on the full key's address: a suffix, and a prefix
                # longer than the key-only span
                if fs.match_address(pk) != f:
                    continue
                found.append(Found(off, b, pk, f))
                if len(found) == quota:
                    break
    finally:
        eng.close()
    found.sort(key=lambda h: h.offset)
    return found[:quota], examined, advances


UNLIMITED = 0xFFFFFFFF


def search_lease(device, root: bytes, first_block: int, blocks: int, filters, report, keep_going=None,
                 max_steps=None, rank: int = 0, world: int = 1, **batch_shape):
    """A worker's leased range (worker::search, src/worker/run.rs:167-238) on
    one GPU: blocks first_block .. first_block + blocks - 1 of `root`, each
    searched from its own seed (block_seed, src/run.rs:211-221), all of them
    at once in the batched engine, until `keep_going()` says stop or
    `max_steps` steps have run.

    Every find is handed to ``report(block, offset)`` as soon as its step
    ends, already confirmed and re-derived on the host: positions are what
    cross the wire, as in the reference. Within a block, finds come in offset
    order. ``report`` returns whether to go on (the reference's callback does
    the same). Returns the number of steps run.

    With one process per GPU, rank ``rank`` of ``world`` takes its share of
    the blocks (``shard.lease_blocks``): the shares are disjoint, and nothing
    crosses between the GPUs."""
    from . import batch as B
    from . import shard

    mine = shard.lease_blocks(first_block, blocks, rank, world)
    b = B.Batch(device, max_searches=max(len(mine), 1), **batch_shape)
    try:
        for blk in mine:
            b.admit(blk, key.block_seed(root, blk), filters, UNLIMITED)
        steps = 0
        while (keep_going is None or keep_going()) and (max_steps is None or steps < max_steps):
            hits = b.step()
            steps += 1
            for h in hits:
                if not report(h.search_id, h.offset):
                    return steps
        return steps
    finally:
        b.close()
