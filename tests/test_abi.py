"""The C ABI library loads and exports every symbol include/*.h declares."""
import ctypes
import glob
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(og_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(native):
    lib = ctypes.CDLL(native._native.LIB_PATH)
    names = declared_functions()
    assert len(names) > 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_exports_are_only_the_c_abi(native):
    out = subprocess.run(["nm", "-D", "--defined-only", native._native.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and l.split()[-1].startswith("og_")}
    assert exported == declared_functions()


def test_no_device_is_an_ordinary_outcome(native):
    """cuda::look (src/gpu/cuda.rs:35-77): no device is a status, not a crash."""
    n = ctypes.c_int(-1)
    err = native._native.errbuf()
    rc = native._native.lib.og_device_count(ctypes.byref(n), err, 512)
    if rc == 0:
        assert n.value >= 1
    else:
        assert native._native.STATUS[rc] == "OG_E_NODEVICE"
        assert n.value == 0
        assert native.gpu.look() == []


def test_resident_lanes_checks_arguments_before_the_device(native):
    """og_engine_resident_lanes refuses a bad scheme or block as OG_E_ARG
    whether or not a device is present; without one it reports a status."""
    n = ctypes.c_uint32(0)
    err = native._native.errbuf()
    L = native._native.lib
    assert native._native.STATUS[L.og_engine_resident_lanes(0, 7, 128, ctypes.byref(n), err, 512)] == "OG_E_ARG"
    assert native._native.STATUS[L.og_engine_resident_lanes(0, 0, 100, ctypes.byref(n), err, 512)] == "OG_E_ARG"
    assert native._native.STATUS[L.og_engine_resident_lanes(0, 0, 128, None, err, 512)] == "OG_E_ARG"
    rc = L.og_engine_resident_lanes(0, 0, 128, ctypes.byref(n), err, 512)
    if native.gpu.look():
        assert rc == 0 and n.value % 128 == 0 and n.value > 0
    else:
        assert rc != 0 and native._native.STATUS[rc] in ("OG_E_DEVICE", "OG_E_NODEVICE")


def test_engine_without_device_reports_status(native, oracle):
    import pytest

    if native.gpu.look():
        pytest.skip("a device is present; covered by the gpu tests")
    start = oracle.scalar_base_mult(oracle.secret_scalar(bytes(32)))
    with pytest.raises(native._native.OgError) as e:
        native.gpu.Engine(0, start, threads=128, bitmap=[0] * 1024, bitmap_bits=16)
    assert e.value.status == "OG_E_NODEVICE"


def test_product_does_not_reference_the_oracle():
    """The product (package and C++/CUDA sources) never imports or loads the oracle."""
    pat = re.compile(r"(from|import)\s+oracle\b|liboracle|oracle/")
    for path in glob.glob(os.path.join(ROOT, "onion_gen_b200", "**", "*"), recursive=True):
        if os.path.isfile(path) and path.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
            assert not pat.search(open(path, errors="replace").read()), path


def test_batch_and_engine_shapes_are_checked_before_the_device(native, oracle):
    """Shape fields that need no device are refused as OG_E_ARG whether or not
    a device is present: the batch's half, max_half, inflight and graph mode,
    and the engine's lanes per thread (1 or 2 for the paired scheme, 1 for
    the chain)."""
    N = native._native
    err = N.errbuf()
    h = ctypes.c_void_p()
    for cfg in (N.BatchConfig(half=4096), N.BatchConfig(half=256, max_half=4096), N.BatchConfig(inflight=3),
                N.BatchConfig(graph=3)):
        rc = N.lib.og_batch_new(0, ctypes.byref(cfg), ctypes.byref(h), err, 512)
        assert N.STATUS[rc] == "OG_E_ARG", err.value
    start = oracle.scalar_base_mult(oracle.secret_scalar(bytes(32)))
    for cfg in (N.EngineConfig(N.SCHEME_PAIRED, 64, 256, 1, 128, 1, 0, 3),
                N.EngineConfig(N.SCHEME_CHAIN, 64, 256, 1, 128, 1, 0, 2)):
        rc = N.lib.og_engine_new_config(0, start, ctypes.byref(cfg), None, 0, 0, ctypes.byref(h), err, 512)
        assert N.STATUS[rc] == "OG_E_ARG", err.value
