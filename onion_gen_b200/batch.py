"""The batched engine: many searches advancing together on one device.

    b = Batch(device=0)
    b.admit(search_id, seed, ["abcd", "efg2"], quota=4)
    while b.running():
        hits = b.step()            # verified hits found in this step
    b.results(search_id)           # the first `quota` hits in offset order

Each step replays one captured CUDA graph: lane initialisation, one
persistent search kernel over every search's lanes, and the device-side
exact match; every hit is re-derived on the host before it counts. Two
steps are in flight by default: ``step()`` launches the next one before it
collects the oldest. A search's result does not depend on what else runs
beside it, nor on its inversion batch (``max_half`` lets long searches run
at a larger one).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _native as N


@dataclass(frozen=True)
class Hit:
    search_id: int
    offset: int
    packed: bytes
    public_key: bytes
    filter: int


STEP_ROOM = 1 << 20


def _hit(h: N.BatchHit) -> Hit:
    return Hit(h.search_id, h.offset, bytes(h.packed), bytes(h.public_key), h.filter)


class Batch:
    def __init__(self, device=0, half=0, slots=0, rounds=0, max_searches=0, max_hits=0, graph=True, memory_budget=0,
                 grid=0, max_half=0, inflight=0):
        ordinal = getattr(device, "ordinal", device)
        cfg = N.BatchConfig(half, slots, rounds, max_searches, max_hits, 1 if graph else 2, grid, memory_budget,
                            max_half, inflight)
        h = C.c_void_p()
        err = N.errbuf()
        N.check(N.lib.og_batch_new(int(ordinal), C.byref(cfg), C.byref(h), err, 512), err)
        self._h = h
        # verified hits one step returns: at most the quotas of the running
        # searches, far below the device's room for exact hits; a step with
        # more fails with OG_E_CAPACITY (the batch keeps them in results())
        self._room = min(N.lib.og_batch_room(h), STEP_ROOM)
        self._buf = (N.BatchHit * self._room)()

    def close(self):
        if getattr(self, "_h", None):
            N.lib.og_batch_free(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def shape(self) -> N.BatchConfig:
        c = N.BatchConfig()
        N.lib.og_batch_shape(self._h, C.byref(c))
        return c

    def admit(self, search_id: int, seed: bytes, prefixes, quota: int) -> None:
        err = N.errbuf()
        text = "\n".join(prefixes).encode()
        N.check(N.lib.og_batch_admit(self._h, search_id, bytes(seed), text, quota, err, 512), err)

    def step(self):
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_batch_step(self._h, self._buf, self._room, C.byref(n), err, 512), err)
        return [_hit(self._buf[i]) for i in range(n.value)]

    def status(self, search_id: int) -> N.SearchStatus:
        st = N.SearchStatus()
        rc = N.lib.og_batch_status(self._h, search_id, C.byref(st))
        if rc:
            raise N.OgError(rc, f"search {search_id}")
        return st

    def results(self, search_id: int):
        st = self.status(search_id)
        room = max(1, min(st.quota, st.hits))
        buf = (N.BatchHit * room)()
        n = C.c_size_t()
        rc = N.lib.og_batch_results(self._h, search_id, buf, room, C.byref(n))
        if rc:
            raise N.OgError(rc, f"search {search_id}")
        return [_hit(buf[i]) for i in range(n.value)]

    def retire(self, search_id: int) -> None:
        rc = N.lib.og_batch_retire(self._h, search_id)
        if rc:
            raise N.OgError(rc, f"search {search_id}")

    def counts(self):
        a, r = C.c_size_t(), C.c_size_t()
        N.lib.og_batch_counts(self._h, C.byref(a), C.byref(r))
        return a.value, r.value

    def running(self) -> int:
        return self.counts()[1]

    def last_step_ms(self) -> float:
        return N.lib.og_batch_last_step_ms(self._h)

    def last_step_candidates(self) -> int:
        return N.lib.og_batch_last_step_candidates(self._h)

    def last_step_launches(self) -> int:
        return N.lib.og_batch_last_step_launches(self._h)

    def plant_mismatch(self, search_id: int) -> None:
        """Tests only: the next hit of the search the host verifies counts as
        one that did not re-derive (the search then ends with OG_E_VERIFY)."""
        rc = N.lib.og_batch_plant_mismatch(self._h, search_id)
        if rc:
            raise N.OgError(rc, f"search {search_id}")

    def memory(self):
        u, b = C.c_uint64(), C.c_uint64()
        N.lib.og_batch_memory(self._h, C.byref(u), C.byref(b))
        return u.value, b.value


def tune(device=0, searches: int = 0, max_step_ms: float = 0.0):
    """og_batch_tune: times the batch over inversion batch, slot pool and grid,
    records the fastest shape (within ``max_step_ms`` of device time a step)
    in tuning.yaml and returns (BatchConfig, keys/s). A Batch created with
    half, slots, rounds and grid all 0 then runs that shape."""
    ordinal = getattr(device, "ordinal", device)
    cfg = N.BatchConfig()
    rate = C.c_double()
    err = N.errbuf()
    N.check(N.lib.og_batch_tune(int(ordinal), searches, max_step_ms, C.byref(cfg), C.byref(rate), err, 512), err)
    return cfg, rate.value
