"""ctypes binding of libonion_gen_b200.so (the C ABI in include/onion_gen_b200.h).

The library is built in-tree (``python onion_gen_b200/build.py``). There is no
fallback: if it is missing or does not load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ONION_GEN_B200_LIB") or os.path.join(HERE, "libonion_gen_b200.so")

OG_OK = 0
STATUS = {
    0: "OG_OK",
    1: "OG_E_ARG",
    2: "OG_E_NODEVICE",
    3: "OG_E_DEVICE",
    4: "OG_E_NOMEM",
    5: "OG_E_OVERFLOW",
    6: "OG_E_CAPACITY",
    7: "OG_E_FILTER",
    8: "OG_E_STATE",
    9: "OG_E_TIMEOUT",
    10: "OG_E_VERIFY",
}
SCHEME_PAIRED = 0
SCHEME_CHAIN = 1


class OgError(RuntimeError):
    """A nonzero og_status with its message."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.status = STATUS.get(code, str(code))
        super().__init__(f"{self.status}: {message}")


class Survivor(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("packed", C.c_uint8 * 32)]


class Match(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("packed", C.c_uint8 * 32), ("filter", C.c_uint32), ("pad", C.c_uint32)]


class EngineConfig(C.Structure):
    _fields_ = [
        ("scheme", C.c_uint32),
        ("half", C.c_uint32),
        ("lanes", C.c_uint32),
        ("rounds", C.c_uint32),
        ("block", C.c_uint32),
        ("dump", C.c_uint32),
        ("room", C.c_uint32),
        ("lanes_per_thread", C.c_uint32),
    ]


class BatchConfig(C.Structure):
    _fields_ = [
        ("half", C.c_uint32),
        ("slots", C.c_uint32),
        ("rounds", C.c_uint32),
        ("max_searches", C.c_uint32),
        ("max_hits", C.c_uint32),
        ("graph", C.c_uint32),
        ("grid", C.c_uint32),
        ("memory_budget", C.c_uint64),
        ("max_half", C.c_uint32),
        ("inflight", C.c_uint32),
    ]


class BatchHit(C.Structure):
    _fields_ = [
        ("search_id", C.c_uint64),
        ("offset", C.c_uint64),
        ("packed", C.c_uint8 * 32),
        ("public_key", C.c_uint8 * 32),
        ("filter", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class SearchStatus(C.Structure):
    _fields_ = [
        ("windows", C.c_uint64),
        ("candidates", C.c_uint64),
        ("hits", C.c_uint64),
        ("lanes", C.c_uint32),
        ("quota", C.c_uint32),
        ("done", C.c_uint32),
        ("filters", C.c_uint32),
        ("table_bytes", C.c_uint64),
        ("status", C.c_uint32),
        ("half", C.c_uint32),
    ]


class ServeConfig(C.Structure):
    _fields_ = [("batch", BatchConfig), ("max_running", C.c_uint32), ("reserved", C.c_uint32)]


class ServeDone(C.Structure):
    _fields_ = [
        ("request_id", C.c_uint64),
        ("arrival_ns", C.c_uint64),
        ("admit_ns", C.c_uint64),
        ("done_ns", C.c_uint64),
        ("candidates", C.c_uint64),
        ("hits", C.c_uint32),
        ("status", C.c_uint32),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("candidates", C.c_uint64),
        ("device_ms", C.c_double),
        ("queued", C.c_uint64),
        ("running", C.c_uint64),
        ("completed", C.c_uint64),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python onion_gen_b200/build.py` "
            "(there is no CPU fallback for the device engine)"
        )
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    B = C.c_char_p
    SZ = C.c_size_t
    U32, U64 = C.c_uint32, C.c_uint64
    I = C.c_int

    def sig(name, res, args):
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args

    sig("og_device_count", I, [C.POINTER(I), B, SZ])
    sig("og_device_info", I, [I, B, SZ, C.POINTER(U64), C.POINTER(I), B, SZ])
    sig("og_engine_new", I, [I, B, U32, P, SZ, U32, I, C.POINTER(P), B, SZ])
    sig("og_engine_new_config", I, [I, B, C.POINTER(EngineConfig), P, SZ, U32, C.POINTER(P), B, SZ])
    sig("og_engine_threads", U32, [P])
    sig("og_engine_batch", U64, [P])
    sig("og_engine_room", SZ, [P])
    sig("og_engine_shape", None, [P, C.POINTER(EngineConfig)])
    sig("og_engine_resident_lanes", I, [I, U32, U32, C.POINTER(U32), B, SZ])
    sig("og_engine_advance", I, [P, P, SZ, C.POINTER(SZ), B, SZ])
    sig("og_engine_launch", I, [P, B, SZ])
    sig("og_engine_collect", I, [P, P, SZ, C.POINTER(SZ), B, SZ])
    sig("og_engine_launch_matches", I, [P, B, SZ])
    sig("og_engine_collect_matches", I, [P, P, SZ, C.POINTER(SZ), B, SZ])
    sig("og_engine_collect_matches_view", I, [P, C.POINTER(P), C.POINTER(SZ), B, SZ])
    sig("og_engine_last_kernel_ms", C.c_float, [P])
    sig("og_engine_match_on_device", I, [P, P, B, SZ])
    sig("og_engine_new_filters", I, [I, B, P, P, C.POINTER(P), B, SZ])
    sig("og_engine_advance_matches", I, [P, P, SZ, C.POINTER(SZ), B, SZ])
    sig("og_engine_free", None, [P])
    sig("og_batch_new", I, [I, C.POINTER(BatchConfig), C.POINTER(P), B, SZ])
    sig("og_batch_admit", I, [P, U64, B, B, U32, B, SZ])
    sig("og_batch_tune", I, [I, U32, C.c_float, C.POINTER(BatchConfig), C.POINTER(C.c_double), B, SZ])
    sig("og_batch_shape", None, [P, C.POINTER(BatchConfig)])
    sig("og_batch_step", I, [P, P, SZ, C.POINTER(SZ), B, SZ])
    sig("og_batch_room", SZ, [P])
    sig("og_batch_status", I, [P, U64, C.POINTER(SearchStatus)])
    sig("og_batch_results", I, [P, U64, P, SZ, C.POINTER(SZ)])
    sig("og_batch_retire", I, [P, U64])
    sig("og_batch_counts", None, [P, C.POINTER(SZ), C.POINTER(SZ)])
    sig("og_batch_last_step_ms", C.c_float, [P])
    sig("og_batch_last_step_candidates", U64, [P])
    sig("og_batch_last_step_launches", U32, [P])
    sig("og_batch_memory", None, [P, C.POINTER(U64), C.POINTER(U64)])
    sig("og_batch_plant_mismatch", I, [P, U64])
    sig("og_batch_free", None, [P])
    sig("og_serve_new", I, [I, C.POINTER(ServeConfig), C.POINTER(P), B, SZ])
    sig("og_serve_submit", I, [P, U64, B, B, U32, B, SZ])
    sig("og_serve_poll", I, [P, P, SZ, C.POINTER(SZ)])
    sig("og_serve_results", I, [P, U64, P, SZ, C.POINTER(SZ)])
    sig("og_serve_stats_get", None, [P, C.POINTER(ServeStats)])
    sig("og_serve_now_ns", U64, [])
    sig("og_serve_free", None, [P])
    sig("og_search_noalloc", I, [I, B, U32, U32, U32, P, U32, P, U32, P, P, B, SZ])
    sig("og_measure_int_peak", I, [I, C.POINTER(C.c_double), C.POINTER(C.c_double), B, SZ])
    sig("og_secret_scalar", None, [B, B])
    sig("og_expanded_secret_key", None, [B, B])
    sig("og_expanded_secret_at_offset", I, [B, U64, B])
    sig("og_scalar_base_mult", None, [B, B])
    sig("og_pack", None, [B, B])
    sig("og_address", None, [B, B])
    sig("og_block_seed", None, [B, U64, B])
    sig("og_check_hit", I, [B, U64, B, B, B])
    sig("og_filters_new", I, [B, U32, C.POINTER(P), B, SZ])
    sig("og_filters_count", SZ, [P])
    sig("og_filters_text", I, [P, SZ, B, SZ])
    sig("og_filters_bits", U32, [P])
    sig("og_filters_words", SZ, [P, C.POINTER(C.POINTER(U64))])
    sig("og_filters_occupancy", C.c_double, [P])
    sig("og_filters_match_probability", C.c_double, [P])
    sig("og_filters_match", C.c_long, [P, B])
    sig("og_filters_match_many", SZ, [P, P, SZ, SZ, P])
    sig("og_filters_prefix_count", SZ, [P])
    sig("og_filters_suffix_bits", U32, [P])
    sig("og_filters_suffix_words", SZ, [P, C.POINTER(C.POINTER(U64))])
    sig("og_filters_match_address", C.c_long, [P, B])
    sig("og_filters_free", None, [P])
    return L


lib = _load()


def errbuf():
    return C.create_string_buffer(512)


def check(code: int, err) -> None:
    if code != OG_OK:
        raise OgError(code, err.value.decode(errors="replace"))
