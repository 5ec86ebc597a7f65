"""Builds libonion_gen_b200.so in-tree for sm_100a.

Device code is compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``;
host C++ with nvcc as well (so one toolchain links everything). Objects go to
``onion_gen_b200/_build/`` and are rebuilt when a source or header is newer.

    python onion_gen_b200/build.py          # build if stale
    python onion_gen_b200/build.py --force  # rebuild everything
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libonion_gen_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]


def sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    return cu, cpp


def headers():
    return (
        glob.glob(os.path.join(CSRC, "*.cuh"))
        + glob.glob(os.path.join(CSRC, "host", "*.h"))
        + glob.glob(os.path.join(ROOT, "include", "*.h"))
    )


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < hdr_mtime


def _compile(src, obj, is_cu, verbose, extra=()):
    cmd = [NVCC] + COMMON + list(extra)
    if is_cu:
        cmd += ARCH + ["-lineinfo", "-Xptxas", "-v"] if verbose else ARCH + ["-lineinfo"]
    else:
        cmd += ["-x", "c++", "-Wno-deprecated-gpu-targets"]
    cmd += ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra=(), lib=None, out=None) -> str:
    """Builds the library (``lib``, objects in ``out``) with optional extra nvcc flags."""
    lib = lib or LIB
    out = out or OUT
    os.makedirs(out, exist_ok=True)
    cu, cpp = sources()
    hdr = max((os.path.getmtime(h) for h in headers()), default=0)
    jobs = []
    objs = []
    for src in cu + cpp:
        rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
        obj = os.path.join(out, rel + ".o")
        objs.append(obj)
        if force or _stale(obj, src, hdr):
            jobs.append((src, obj, src.endswith(".cu")))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, c, verbose, extra) for s, o, c in jobs]
            for f in futs:
                logs.append(f.result())
    if jobs or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        for l in logs:
            if l:
                print(l)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
