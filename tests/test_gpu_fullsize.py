"""Configs 2 and 3 over their full 2^32 candidates (runs on a B200: -m gpu).

At this size the oracle would take minutes, so these tests check what holds
at any size, over the whole range:
- every survivor is the key of its offset, re-derived on the host from the
  offset alone (src/run.rs:1089-1104);
- offsets are unique multiples of 8 inside [8, 8 * 2^32];
- every survivor's slot is set in the index, and their number is within
  Poisson bounds of what the index lets through;
- the device's exact match equals the host's match of every survivor
  (src/filter.rs:2194-2213) over the same range.
The oracle pins the same engines on their first 2^24 candidates
(test_gpu_engine.py).
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import gpu, key, workloads

pytestmark = pytest.mark.gpu

FULL = 1 << 32


def over_range(eng, get, n=FULL):
    """Advances until n candidates are covered; keeps the records whose
    offset is at most 8 n (offsets run from 8 upwards)."""
    parts, covered = [], 0
    while covered < n:
        rec = get()
        covered += eng.batch()
        keep = rec[0] <= 8 * n
        parts.append([a[keep] for a in rec])
    return [np.concatenate([p[i] for p in parts]) for i in range(len(parts[0]))]


def match_all(fs, packed):
    """FilterSet.match_many over row chunks on every host core (the library
    call releases the GIL and only reads the set)."""
    k = max(1, min(32, os.cpu_count() or 1))
    with ThreadPoolExecutor(k) as ex:
        parts = list(ex.map(fs.match_many, np.array_split(packed, k)))
    return np.concatenate(parts)


def all_distinct(a):
    s = np.sort(a)
    return bool((s[1:] != s[:-1]).all())


def slots_of(packed, bits):
    head = packed[:, :4].astype(np.uint32)
    h32 = (head[:, 0] << 24) | (head[:, 1] << 16) | (head[:, 2] << 8) | head[:, 3]
    return (h32 >> np.uint32(32 - bits)).astype(np.uint64)


def test_config2_full_range(device):
    """Config 2: seed LE32(0), one 6-symbol prefix on a 16-bit index, 2^32
    candidates at the bench's shape."""
    seed = workloads.seed(0)
    start = key.start_point(seed)
    prefix = workloads.config2_prefix()
    fs = F.FilterSet.parse_all([prefix])
    words, bits = fs.index_words()
    assert bits == 16
    with gpu.Engine(device, start, bitmap=words, bitmap_bits=bits) as eng:
        offs, keys = over_range(eng, eng.advance_raw)
    assert all_distinct(offs)
    assert (offs % 8 == 0).all() and offs.min() >= 8 and offs.max() <= 8 * FULL
    slot = slots_of(keys, bits)
    assert (((words[slot >> 6] >> (slot & 63)) & 1) == 1).all()
    mu = FULL * fs.occupancy()  # one slot of 2^16: 65,536
    assert abs(len(offs) - mu) < 6 * mu**0.5
    for o, k in zip(offs, keys):
        pk, _ = key.check_hit(seed, int(o), bytes(k))
    m = fs.match_many(keys)
    host = sorted(zip(offs[m >= 0].tolist(), m[m >= 0].tolist()))
    with gpu.Engine(device, start, filters=fs) as eng:
        moffs, mkeys, mfil = over_range(eng, eng.advance_matches_raw)
    assert sorted(zip(moffs.tolist(), mfil.tolist())) == host
    for o, k in zip(moffs, mkeys):
        pk, _ = key.check_hit(seed, int(o), bytes(k))
        assert key.address(pk).startswith(prefix)


def test_config3_full_range_device_match_equals_host(device):
    """Config 3: 10,000 prefixes of 3..8 symbols on a 24-bit index (~5 % of
    candidates survive and match), 2^32 candidates. Two engines over the
    same range, advance by advance: one returns the bitmap survivors, the
    other the device's exact matches, which must equal the host's match of
    those survivors exactly."""
    seed = workloads.seed(0)
    start = key.start_point(seed)
    fs = F.FilterSet.parse_all(workloads.config3_prefixes())
    words, bits = fs.index_words()
    assert bits == 24
    lanes = max(128, gpu.resident_lanes(device) // 2 // 128 * 128)
    cfg = N.EngineConfig(N.SCHEME_PAIRED, 2048, lanes, 1, 128, 0, 0)
    rng = np.random.default_rng(3)
    survivors = matches = covered = 0
    with gpu.Engine(device, start, bitmap=words, bitmap_bits=bits, config=cfg) as a, \
            gpu.Engine(device, start, filters=fs, config=cfg) as b:
        assert a.batch() == b.batch()
        while covered < FULL:
            so, sk = a.advance_raw()
            mo, mk, mf = b.advance_matches_raw()
            covered += a.batch()
            keep, mkeep = so <= 8 * FULL, mo <= 8 * FULL
            so, sk = so[keep], sk[keep]
            mo, mk, mf = mo[mkeep], mk[mkeep], mf[mkeep]
            hm = match_all(fs, sk)
            host = np.sort((so[hm >= 0] << np.uint64(14)) | hm[hm >= 0].astype(np.uint64))
            dev = np.sort((mo << np.uint64(14)) | mf.astype(np.uint64))
            assert np.array_equal(host, dev)
            assert all_distinct(so)
            for i in rng.choice(len(mo), size=min(32, len(mo)), replace=False):
                key.check_hit(seed, int(mo[i]), bytes(mk[i]))
            survivors += len(so)
            matches += len(mo)
    assert covered >= FULL
    # about 5 % of the key space is covered by the prefixes and the index
    assert 0.04 * FULL < matches <= survivors < 0.07 * FULL
