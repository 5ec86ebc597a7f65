"""The device engine, shaped like onion-gen's ``gpu::Engine`` (src/gpu/mod.rs).

    engine = Engine(device=0, start=point, threads=0, bitmap=words, bitmap_bits=bits)
    engine.threads()   # lanes in flight          (src/gpu/mod.rs:452)
    engine.batch()     # candidates per advance   (src/gpu/mod.rs:461)
    engine.advance()   # -> list[Survivor]        (src/gpu/mod.rs:470)

A ``Survivor`` is ``(offset, packed)``: the scalar delta from the start point's
scalar and the packed key with the sign bit clear (src/gpu/mod.rs:113-119).
Everything runs through ``libonion_gen_b200.so``; errors raise ``OgError``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import OgError  # noqa: F401  (re-exported)


@dataclass(frozen=True)
class Survivor:
    offset: int
    packed: bytes


@dataclass(frozen=True)
class Device:
    index: int
    ordinal: int
    name: str
    memory: int
    sms: int


def look():
    """Devices the CUDA driver reports (cuda::look, src/gpu/cuda.rs:35-77).

    Returns a list of ``Device``; an empty list when there is no driver or no
    device (an ordinary outcome, not an error)."""
    n = C.c_int()
    err = N.errbuf()
    if N.lib.og_device_count(C.byref(n), err, 512) != N.OG_OK:
        return []
    out = []
    for i in range(n.value):
        name = C.create_string_buffer(256)
        mem = C.c_uint64()
        sms = C.c_int()
        if N.lib.og_device_info(i, name, 256, C.byref(mem), C.byref(sms), err, 512) == N.OG_OK:
            out.append(Device(len(out), i, name.value.decode(), mem.value, sms.value))
    return out


def resident_lanes(device, scheme=None, block=128):
    """Lanes one wave of the search kernel holds on ``device``: resident
    blocks per SM x SMs x ``block``. The paired kernel runs exactly this
    many threads; its lanes are taken a block at a time."""
    n = C.c_uint32()
    err = N.errbuf()
    scheme = N.SCHEME_PAIRED if scheme is None else scheme
    N.check(N.lib.og_engine_resident_lanes(device.ordinal, scheme, block, C.byref(n), err, 512), err)
    return n.value


def _words(bitmap):
    if bitmap is None:
        return None, 0
    arr = np.ascontiguousarray(np.asarray(bitmap, dtype=np.uint64))
    return arr, arr.size


class Engine:
    """One search on one device (gpu::Engine::new, src/gpu/mod.rs:346-413).

    ``start`` is the chain's first point as 128 bytes (X, Y, Z, T) — e.g.
    ``key.start_point(seed)``. ``threads=0`` takes the shape from tuning.yaml,
    or times the candidates and records the fastest. ``config`` (an
    ``EngineConfig``) names an explicit shape instead. ``filters`` (a
    ``filter.FilterSet``, prefixes and suffixes) builds both bitmaps from the
    set and turns the device match on (og_engine_new_filters); ``bitmap`` is
    then ignored.
    """

    def __init__(self, device=0, start=None, threads=0, bitmap=None, bitmap_bits=0, retune=False, config=None,
                 filters=None):
        ordinal = device.ordinal if isinstance(device, Device) else int(device)
        if start is None or len(start) != 128:
            raise ValueError("start must be a 128-byte point (X, Y, Z, T)")
        self._words, nwords = _words(bitmap)
        ptr = self._words.ctypes.data if self._words is not None else None
        h = C.c_void_p()
        err = N.errbuf()
        if filters is not None:
            # og_engine_new_filters: both bitmaps from the set, device match on
            cfgp = C.byref(config) if config is not None else None
            rc = N.lib.og_engine_new_filters(ordinal, bytes(start), filters._h, cfgp, C.byref(h), err, 512)
        elif config is not None:
            rc = N.lib.og_engine_new_config(
                ordinal, bytes(start), C.byref(config), ptr, nwords, bitmap_bits, C.byref(h), err, 512
            )
        else:
            rc = N.lib.og_engine_new(
                ordinal, bytes(start), threads, ptr, nwords, bitmap_bits, 1 if retune else 0, C.byref(h), err, 512
            )
        N.check(rc, err)
        self._h = h
        self._room = N.lib.og_engine_room(h)
        self._buf = (N.Survivor * max(self._room, 1))()
        if filters is not None:
            self._mbuf = (N.Match * max(self._room, 1))()

    def close(self):
        if getattr(self, "_h", None):
            N.lib.og_engine_free(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def threads(self) -> int:
        return N.lib.og_engine_threads(self._h)

    def batch(self) -> int:
        return N.lib.og_engine_batch(self._h)

    def room(self) -> int:
        return self._room

    def shape(self) -> N.EngineConfig:
        c = N.EngineConfig()
        N.lib.og_engine_shape(self._h, C.byref(c))
        return c

    def last_kernel_ms(self) -> float:
        return N.lib.og_engine_last_kernel_ms(self._h)

    def advance_raw(self):
        """advance() as numpy arrays: (offsets uint64[n], packed uint8[n, 32])."""
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_engine_advance(self._h, self._buf, self._room, C.byref(n), err, 512), err)
        k = n.value
        raw = np.frombuffer(self._buf, dtype=np.uint8, count=k * 40).reshape(k, 40)
        offsets = raw[:, :8].copy().view(np.uint64).reshape(k)
        return offsets, raw[:, 8:40].copy()

    def advance(self):
        offsets, packed = self.advance_raw()
        return [Survivor(int(o), bytes(p)) for o, p in zip(offsets, packed)]

    def launch(self):
        """og_engine_launch: enqueue one advance and return at once (at most
        two in flight)."""
        err = N.errbuf()
        N.check(N.lib.og_engine_launch(self._h, err, 512), err)

    def collect_raw(self):
        """og_engine_collect: the oldest launched advance's survivors, as
        advance_raw returns them."""
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_engine_collect(self._h, self._buf, self._room, C.byref(n), err, 512), err)
        return self._survivors(n.value)

    def _survivors(self, k):
        raw = np.frombuffer(self._buf, dtype=np.uint8, count=k * 40).reshape(k, 40)
        offsets = raw[:, :8].copy().view(np.uint64).reshape(k)
        return offsets, raw[:, 8:40].copy()

    def match_on_device(self, filters):
        """Exact match on the device from now on (og_engine_match_on_device):
        ``filters`` is the ``filter.FilterSet`` whose index_words this engine
        was created with."""
        err = N.errbuf()
        N.check(N.lib.og_engine_match_on_device(self._h, filters._h, err, 512), err)
        self._mbuf = (N.Match * max(self._room, 1))()

    def advance_matches_raw(self):
        """One advance returning only exact matches, as numpy arrays:
        (offsets uint64[n], packed uint8[n, 32], filter index uint32[n])."""
        if getattr(self, "_mbuf", None) is None:
            raise N.OgError(8, "match_on_device() has not been called")
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_engine_advance_matches(self._h, self._mbuf, self._room, C.byref(n), err, 512), err)
        return self._matches(n.value)

    def launch_matches(self):
        """og_engine_launch_matches: enqueue one advance with the device match."""
        err = N.errbuf()
        N.check(N.lib.og_engine_launch_matches(self._h, err, 512), err)

    def collect_matches_raw(self):
        """og_engine_collect_matches: the oldest launched advance's matches."""
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_engine_collect_matches(self._h, self._mbuf, self._room, C.byref(n), err, 512), err)
        return self._matches(n.value)

    def collect_matches_view(self):
        """og_engine_collect_matches_view: the oldest launched advance's
        matches where the engine keeps them (its pinned host memory), as a
        ctypes array of ``Match`` valid until the next collect; no copy."""
        p = C.c_void_p()
        n = C.c_size_t()
        err = N.errbuf()
        N.check(N.lib.og_engine_collect_matches_view(self._h, C.byref(p), C.byref(n), err, 512), err)
        if n.value == 0:
            return (N.Match * 0)()
        return (N.Match * n.value).from_address(p.value)

    def collect_matches_view_raw(self):
        """collect_matches_view copied out as (offsets, packed, filters) arrays."""
        view = self.collect_matches_view()
        return self._matches(len(view), view)

    def _matches(self, k, buf=None):
        raw = np.frombuffer(self._mbuf if buf is None else buf, dtype=np.uint8, count=k * 48).reshape(k, 48)
        offsets = raw[:, :8].copy().view(np.uint64).reshape(k)
        filters = raw[:, 40:44].copy().view(np.uint32).reshape(k)
        return offsets, raw[:, 8:40].copy(), filters
