"""Benchmark of the key-search hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the plain GPU search at scale): one search from the base scalar of
seed LE32(0), one 6-symbol base32 prefix from splitmix64(2), a 16-bit prefix
index, and 2^32 candidates per step (rounded up to whole advances; the
candidates actually examined are what is counted). Inputs are synthetic.

One JSON line on rank 0:
  value       keys/s over the timed steps, device time (CUDA events on the
              engine's stream around every kernel launch), max over ranks
  e2e         keys/s through the C ABI as a caller uses it: engine creation
              (host precompute, H2D of the start point, tables and bitmap),
              every advance (D2H of the survivors) and the host's exact match
              and independent re-derivation of every hit, wall clock
  roofline    integer-multiply bound: partial products/s achieved by the
              search kernel against the measured multiply-add issue rate
  cpu_baseline the oracle's restatement of the reference's paired CPU engine
              (src/pairs.rs, batch 8192 as src/run.rs uses) on every host core

--impl reference times that CPU engine alone (the reference's GPU engine is
Rust compiled to PTX by a nightly toolchain that is not available here).
Multi-GPU: one process per GPU; each rank searches its own disjoint offset
range (no collective on the data path); weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CANDIDATES_PER_STEP = 1 << 32
HALF = 256
CPU_HALF = 4096  # PairEngine::new(8192) (src/run.rs:601, src/batch.rs:32)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--case", default="full", choices=["full", "small"],
                   help="small: the profiling case, three one-round advances of the plain engine")
    p.add_argument("--half", type=int, default=HALF)
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """Samples nvidia-smi during the timed region."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(s[1]) for s in self.samples if num(s[1])]
        mx = [num(s[2]) for s in self.samples if num(s[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        power = [num(s[3]) for s in self.samples if num(s[3])]
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "power_w_max": max(power) if power else None,
            "samples": len(self.samples),
        }


def cpu_baseline(seconds):
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    O.pair_rate(threads, 0.5, CPU_HALF)  # warm-up round
    rate, examined = O.pair_rate(threads, seconds, CPU_HALF)
    return {
        "value": rate,
        "unit": "keys/s",
        "cores": threads,
        "kind": "port",
        "sample": f"{examined} candidates of the paired CPU engine (batch 8192) with a 16-bit prefix probe, "
        f"{threads} threads x {seconds:.0f} s after one untimed round",
    }


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    seconds = max(1.0, min(10.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        O.pair_rate(threads, seconds, CPU_HALF)
    total, t = 0, 0.0
    for _ in range(args.steps):
        r, ex = O.pair_rate(threads, seconds, CPU_HALF)
        total += ex
        t += ex / r if r else 0
    value = total / t if t else 0.0
    line = {
        "impl": "reference",
        "metric": "keys/s (plain search, 2^32 candidates, one 6-char prefix)",
        "value": value,
        "unit": "keys/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t / max(1, args.steps),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": "config 2 shape on the host: paired CPU engine, seeds per thread, 16-bit prefix probe",
                   "threads": threads},
        "cpu_baseline": {"value": value, "unit": "keys/s", "cores": threads, "kind": "port",
                         "sample": f"{total} candidates, {args.steps} steps of {seconds:.1f} s on {threads} threads"},
        "e2e": {"value": value, "unit": "keys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's GPU engine is Rust->PTX built by a nightly toolchain absent here; its CPU engine "
        "is restated in C (oracle/) and timed instead",
    }
    print(json.dumps(line), flush=True)


def pp_per_candidate(half):
    """Partial products per candidate of the paired round: (21 + 10 half)
    multiplications of 64 and 254 squarings of 36, over 2 half + 1 keys."""
    return ((21 + 10 * half) * 64 + 254 * 36) / (2 * half + 1)


def small_case(args):
    """Three advances of one round each at the default shape: the case the
    ncu summaries under profiles/ are captured on (about 1.6 GB of scratch)."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    dev = gpu.look()[0]
    fs = F.FilterSet.parse_all([workloads.config2_prefix()])
    words, bits = fs.index_words()
    start = key.start_point(workloads.seed(0))
    eng = gpu.Engine(dev, start, bitmap=words, bitmap_bits=bits, config=N.EngineConfig(0, args.half, 0, 1, 128, 0, 0))
    for i in range(3):
        o, _ = eng.advance_raw()
        ms = eng.last_kernel_ms()
        print(f"advance {i}: {len(o)} survivors, kernel {ms:.3f} ms, {eng.batch() / ms * 1e3:.4e} keys/s")


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.case == "small":
        small_case(args)
        return
    rank, world, local = dist_env()
    import ctypes as C

    import numpy as np
    import torch

    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    dev = gpu.look()[local]
    seed = workloads.seed(0)
    prefix = workloads.config2_prefix()
    fs = F.FilterSet.parse_all([prefix])
    words, bits = fs.index_words()
    # rank r searches offsets [r * 2^40 * 8, ...): start = s B + r 2^43 B
    # rank r searches its own range: base scalar s + r 2^43 (offsets below 2^43 never meet)
    scalar = int.from_bytes(key.secret_scalar(seed), "little") + (rank << 43)
    base = key.scalar_base_mult(scalar.to_bytes(32, "little"))

    cfg = N.EngineConfig(N.SCHEME_PAIRED, args.half, 0, 0, 128, 0, 0)
    eng = gpu.Engine(dev, base, bitmap=words, bitmap_bits=bits, config=cfg)
    shape = eng.shape()
    batch = eng.batch()
    advances = -(-CANDIDATES_PER_STEP // batch)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        ms = 0.0
        surv = 0
        for _ in range(advances):
            o, k = eng.advance_raw()
            ms += eng.last_kernel_ms()
            surv += len(o)
        return ms, surv

    for _ in range(args.warmup):
        step()
    barrier()
    dev_ms, survivors = [], 0
    with Clocks(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between steps (outside the kernel events)
            torch.cuda.synchronize()
            ms, s = step()
            dev_ms.append(ms)
            survivors += s
        barrier()
        wall = time.perf_counter() - t0
    total_ms = sum(dev_ms)
    per_rank = np.array([total_ms, wall], dtype=np.float64)
    if pg:
        t = torch.tensor(per_rank, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        per_rank = t.cpu().numpy()
    total_ms, wall = float(per_rank[0]), float(per_rank[1])
    keys = batch * advances * args.steps * world
    value = keys / (total_ms * 1e-3)

    # integer-multiply roofline
    imad = C.c_double()
    mulpp = C.c_double()
    err = N.errbuf()
    N.check(N.lib.og_measure_int_peak(dev.ordinal, C.byref(imad), C.byref(mulpp), err, 512), err)
    w = pp_per_candidate(shape.half)
    achieved = value / world * w
    peak = imad.value / 2.0

    # end to end through the C ABI, host buffers, every hit re-derived
    e2e = None
    if not args.no_e2e:
        h2d = d2h = 0
        hits = 0
        barrier()
        t1 = time.perf_counter()
        for _ in range(max(1, args.steps // 2)):
            e = gpu.Engine(dev, base, bitmap=words, bitmap_bits=bits, config=cfg)
            h2d += 128 + words.nbytes + shape.half * 96
            for _ in range(advances):
                o, k = e.advance_raw()
                d2h += 4 + 48 * len(o)
                for off, packed in zip(o, k):
                    if fs.match_key(bytes(packed)) is not None:
                        key.check_hit(seed, int(off) + (rank << 43), bytes(packed))
                        hits += 1
            e.close()
        barrier()
        e2e_wall = time.perf_counter() - t1
        e2e_steps = max(1, args.steps // 2)
        e2e = {
            "value": batch * advances * e2e_steps * world / e2e_wall,
            "unit": "keys/s",
            "h2d_bytes_per_step": h2d // e2e_steps,
            "d2h_bytes_per_step": d2h // e2e_steps,
            "steps": e2e_steps,
            "hits_verified": hits,
        }

    if rank == 0:
        line = {
            "metric": "keys/s (plain search, 2^32 candidates, one 6-char prefix)",
            "value": value,
            "unit": "keys/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u32",
            "data": "synthetic",
            "config": {
                "workload": "plain search: seed LE32(0), prefix %r (16-bit index), 2^32 candidates per step" % prefix,
                "scheme": "paired",
                "half": shape.half,
                "lanes": shape.lanes,
                "rounds_per_advance": shape.rounds,
                "advances_per_step": advances,
                "candidates_per_step": batch * advances,
                "l2": "flushed between steps (256 MiB write); per-step scratch exceeds L2",
                "parallelism": f"independent ranges x{world}",
            },
            "wall_s": wall,
            "survivors": survivors,
            "gpu_launches": advances * args.steps,
            "roofline": {
                "bound": "int-mul",
                "achieved": achieved,
                "peak": peak,
                "unit": "partial products/s",
                "frac": achieved / peak,
                "traffic": None,
                "per_candidate": w,
                "peak_source": "measured: og_measure_int_peak mad.lo.u32 issue rate / 2 (lo+hi per product)",
                "fe_mul_pp_per_s": mulpp.value,
            },
            "clocks": clocks.summary(),
        }
        if e2e:
            line["e2e"] = e2e
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
