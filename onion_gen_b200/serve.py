"""The serving loop: continuous batching of search requests on one device.

    s = Server(device=0)
    s.submit(request_id, seed, ["abcd"], quota=4)   # from any thread
    for done in s.poll():                          # og_serve_done records
        hits = s.results(done.request_id)

A native worker thread admits queued requests as lanes and device memory
allow, steps the batched engine, and retires each request at the end of the
step that meets its quota. Time-to-find is ``done_ns - arrival_ns``.
"""
from __future__ import annotations

import ctypes as C

from . import _native as N
from .batch import _hit


class Server:
    def __init__(self, device=0, half=0, slots=0, rounds=0, max_searches=0, max_hits=0, graph=True,
                 memory_budget=0, max_running=0, grid=0, max_half=0, inflight=0):
        ordinal = getattr(device, "ordinal", device)
        cfg = N.ServeConfig(N.BatchConfig(half, slots, rounds, max_searches, max_hits, 1 if graph else 2, grid,
                                          memory_budget, max_half, inflight), max_running, 0)
        h = C.c_void_p()
        err = N.errbuf()
        N.check(N.lib.og_serve_new(int(ordinal), C.byref(cfg), C.byref(h), err, 512), err)
        self._h = h
        self._buf = (N.ServeDone * 4096)()

    def close(self):
        if getattr(self, "_h", None):
            N.lib.og_serve_free(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, request_id: int, seed: bytes, prefixes, quota: int) -> None:
        err = N.errbuf()
        N.check(N.lib.og_serve_submit(self._h, request_id, bytes(seed), "\n".join(prefixes).encode(), quota, err, 512),
                err)

    def poll(self):
        out = []
        while True:
            n = C.c_size_t()
            N.lib.og_serve_poll(self._h, self._buf, len(self._buf), C.byref(n))
            out += [self._buf[i] for i in range(n.value)]
            if n.value < len(self._buf):
                return [N.ServeDone.from_buffer_copy(d) for d in out]

    def results(self, request_id: int, quota: int = 64):
        buf = (N.BatchHit * quota)()
        n = C.c_size_t()
        rc = N.lib.og_serve_results(self._h, request_id, buf, quota, C.byref(n))
        if rc:
            raise N.OgError(rc, f"request {request_id}")
        return [_hit(buf[i]) for i in range(n.value)]

    def stats(self) -> N.ServeStats:
        st = N.ServeStats()
        N.lib.og_serve_stats_get(self._h, C.byref(st))
        return st

    @staticmethod
    def now_ns() -> int:
        return N.lib.og_serve_now_ns()
