"""Benchmark of the key-search hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the plain GPU search at scale): one search from the base scalar of
seed LE32(0), one 6-symbol base32 prefix from splitmix64(2), a 16-bit prefix
index, and 2^32 candidates per step (rounded up to whole advances; the
candidates actually examined are what is counted). Inputs are synthetic.

One JSON line on rank 0:
  value       keys/s over the timed steps, device time (CUDA events on the
              engine's stream around every kernel launch), max over ranks
  e2e         keys/s through the C ABI as a caller uses it: one engine for
              the run, its creation (host precompute, H2D of the start point,
              tables and bitmap) and free, every advance (D2H of the
              survivors) and the host's exact match and independent
              re-derivation of every hit, wall clock
  roofline    integer-multiply bound: partial products/s achieved by the
              search kernel against the measured multiply-add issue rate
  cpu_baseline the oracle's restatement of the reference's paired CPU engine
              (src/pairs.rs, batch 8192 as src/run.rs uses) on every host core

  suffix      a suffix search (16 suffixes of 9 symbols) through the filter
              engine: suffix bitmap in the search kernel, full key, sign bit
              and SHA3-256 checksum recomputed on the device for its
              survivors, every match re-derived on the host
  batch_shape the batch's autotuner (og_batch_tune): inversion batch,
              slot pool and grid, the fastest within 8 ms a step; the
              batched and serving legs run that shape
  config3     config 3 (10,000 prefixes of 3..8 symbols, a 24-bit index, 2^32
              candidates a step) with the exact match on the device: kernel
              keys/s and its roofline fraction, and end to end with every
              match copied back and a sample re-derived on the host
  batched     config 4 (all 64 searches, 1..5000 prefixes of 4..7 symbols,
              quota 1..16): the single-search engine one search at a time
              (the run driver's loop), once with the reference-shaped
              constructor's tuned shape and once at half 256, against the
              batched engine (long searches at a larger inversion batch, two
              steps in flight); same results
  serving     config 5 (all 2000 requests, Poisson arrivals at 50/s, 1..200
              prefixes, quota 1..16) through the serving loop under a
              wall-clock cap: p50/p99 time-to-find over all requests, a
              request unfinished at the cap counted at its elapsed time as a
              lower bound (censored)

--impl reference times that CPU engine alone (the reference's GPU engine is
Rust compiled to PTX by a nightly toolchain that is not available here).
Multi-GPU: one process per GPU; each rank searches its own disjoint offset
range (no collective on the data path); weak scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CANDIDATES_PER_STEP = 1 << 32
HALF = 2048
# the plain engine of the batched leg (one search at a time) and the batch's
# profiling case: a short round, so that small searches do not overshoot
SHORT_HALF = 256
# the batch's shape comes from its autotuner, within this much device time a step
BATCH_STEP_CAP_MS = 8.0
CPU_HALF = 4096  # PairEngine::new(8192) (src/run.rs:601, src/batch.rs:32)
# DRAM bytes per candidate of paired_kernel, from the ncu capture of the
# small case (bench.py --case small: half 256, 757,760 lanes, one launch of
# 388,730,880 candidates; dram__bytes_read.sum + dram__bytes_write.sum =
# 24.96 + 25.03 GB), scaled to a launch of the plain line by its candidates:
# the traffic is the Montgomery scratch, 64 B written and 64 B read per
# candidate, whatever the shape, so it grows in proportion.
TRAFFIC_PER_CANDIDATE = 128.6
ALGORITHMIC_BYTES_PER_CANDIDATE = 128


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--case", default="full",
                   choices=["full", "small", "batch-small", "suffix-small", "chain-small", "config3-small"],
                   help="small: the profiling case, three one-round advances of the plain engine; "
                   "batch-small: three steps of the batched engine over the first 16 config-4 searches; "
                   "suffix-small: three advances of a forty-suffix search with the device match; "
                   "chain-small: three advances of the chain scheme at its default shape; "
                   "config3-small: three advances of config 3's 10,000-prefix search at its default shape")
    p.add_argument("--lanes-per-thread", type=int, default=1,
                   help="lanes each thread of the paired search kernel carries in --case small (1 or 2)")
    p.add_argument("--half", type=int, default=0,
                   help=f"inversion batch half-width (default {HALF} for the plain line, 256 for --case small, "
                   f"{SHORT_HALF} for the batch's profiling case)")
    p.add_argument("--suite", default="default",
                   choices=["default", "batched", "serving", "plain", "suffix", "config3"],
                   help="default: the plain line plus the chain, suffix, config-3, batched and serving legs; "
                   "batched / serving / suffix / config3: that leg alone; plain: the plain line only")
    p.add_argument("--batched-cap", type=float, default=float("inf"),
                   help="largest expected work (candidates) of a config-4 search to run (default: all)")
    p.add_argument("--serving-requests", type=int, default=2000)
    p.add_argument("--serving-cap", type=float, default=60.0, help="serving wall-clock cap, seconds")
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


def plain_workload(prefix):
    return "plain search: seed LE32(0), prefix %r (16-bit index), 2^32 candidates per step" % prefix


def config2_search():
    """Config 2's seed, prefix and prefix index for the CPU legs, without the
    product's library: the workload generator loaded from its file and the
    oracle's FilterSet."""
    import importlib.util

    from oracle import oracle as O

    spec = importlib.util.spec_from_file_location("og_workloads", os.path.join(ROOT, "onion_gen_b200", "workloads.py"))
    W = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = W
    spec.loader.exec_module(W)
    prefix = W.config2_prefix()
    fs = O.FilterSet([prefix])
    return W.seed(0), prefix, fs.words(), fs.bits


def cpu_baseline(seconds):
    """The reference's paired CPU engine restated (oracle/), timed the way
    src/estimate.rs:86-117 does: one untimed round, then the median of three
    timed runs on every host thread, each thread on its own sub-range of
    config 2's search with config 2's prefix index. The chain engine
    (src/batch.rs) is timed beside it for context."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    seed, prefix, words, bits = config2_search()
    O.pair_rate_search(threads, 0.5, CPU_HALF, seed, words, bits)  # untimed round
    runs = [O.pair_rate_search(threads, seconds / 3, CPU_HALF, seed, words, bits) for _ in range(3)]
    rates = sorted(r for r, _ in runs)
    examined = sum(ex for _, ex in runs)
    chain, _ = O.chain_rate(threads, min(2.0, seconds / 3), 8192)
    return {
        "value": rates[1],
        "unit": "keys/s",
        "cores": threads,
        "kind": "port",
        "sample": f"{examined} candidates of config 2's search (seed LE32(0), prefix {prefix!r}, its {bits}-bit index) "
        f"by the paired CPU engine (batch 8192), thread t from candidate 2^40 t: median of 3 runs of "
        f"{seconds / 3:.1f} s on {threads} threads after one untimed round",
        "runs": rates,
        "chain_engine_keys_per_s": chain,
    }


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    seconds = max(1.0, min(10.0, 60.0 / max(1, args.steps + args.warmup)))
    seed, prefix, words, bits = config2_search()
    for _ in range(args.warmup):
        O.pair_rate_search(threads, seconds, CPU_HALF, seed, words, bits)
    total, t = 0, 0.0
    for _ in range(args.steps):
        r, ex = O.pair_rate_search(threads, seconds, CPU_HALF, seed, words, bits)
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
        "config": {"workload": plain_workload(prefix), "engine": "paired CPU engine (batch 8192), restated in C",
                   "threads": threads},
        "cpu_baseline": {"value": value, "unit": "keys/s", "cores": threads, "kind": "port",
                         "sample": f"{total} candidates of the search, thread t from candidate 2^40 t: "
                         f"{args.steps} steps of {seconds:.1f} s on {threads} threads"},
        "e2e": {"value": value, "unit": "keys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's GPU engine is Rust->PTX built by a nightly toolchain absent here; its CPU engine "
        "is restated in C (oracle/) and timed instead",
    }
    print(json.dumps(line), flush=True)


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def batch_shape(dev):
    """The batch's autotuner (og_batch_tune): inversion batch, slot pool and
    grid, the fastest within BATCH_STEP_CAP_MS of device time a step."""
    from onion_gen_b200 import batch as B

    t0 = time.perf_counter()
    cfg, rate = B.tune(dev, 64, BATCH_STEP_CAP_MS)
    shape = {"half": cfg.half, "slots": cfg.slots, "grid": cfg.grid, "rounds": cfg.rounds}
    log(f"batch tuner: {shape} at {rate:.4e} keys/s in {time.perf_counter() - t0:.1f} s")
    return shape, {**shape, "tuned_keys_per_s": rate, "step_cap_ms": BATCH_STEP_CAP_MS,
                   "tune_s": time.perf_counter() - t0}


# config-4 searches whose expected work is above this many candidates are
# the "long" ones (two of the 64: 2.4e11 and 4.1e11 expected candidates)
LONG_SEARCH = 2e10


def plain_arm(dev, searches, config, device_match):
    """The run driver's loop (src/run.rs:1036-1074): one engine per search,
    one search at a time, until its quota of verified hits; the survivors
    are matched on the host (FilterSet::match_key, as the reference does)
    or on the device."""
    from onion_gen_b200 import run

    out, examined, launches, per = {}, 0, 0, {}
    t0 = time.perf_counter()
    for s in searches:
        t1 = time.perf_counter()
        found, ex, advances = run.device_search(dev, s.seed, s.prefixes, s.quota, config=config,
                                                device_match=device_match)
        per[s.index] = time.perf_counter() - t1
        out[s.index] = [(h.offset, h.packed) for h in found]
        examined += ex
        launches += 2 * advances + 1
    wall = time.perf_counter() - t0
    long_s = sum(t for i, t in per.items() if searches_by_index(searches)[i].expected_candidates() > LONG_SEARCH)
    return out, {"wall_s": wall, "examined": examined, "examined_per_s": examined / wall, "gpu_launches": launches,
                 "long_searches_wall_s": long_s, "short_searches_wall_s": wall - long_s}


def searches_by_index(searches):
    return {s.index: s for s in searches}


def batched_leg(dev, shape, cap, kernel_rate):
    """Config 4: the plain engine (one engine per search, the run driver's
    loop) against the batched engine, same searches, same results."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import batch as B
    from onion_gen_b200 import gpu, key, workloads

    all_searches = workloads.config4_searches()
    searches = [s for s in all_searches if s.expected_candidates() <= cap]
    # the reference-shaped constructor (og_engine_new, threads = 0) takes its
    # shape from tuning.yaml, timing the candidates once if there is none:
    # that walk runs here, before the clock
    probe = gpu.Engine(dev, key.start_point(workloads.seed(0)), threads=0,
                       bitmap=np.zeros(1024, dtype=np.uint64), bitmap_bits=16)
    tuned = probe.shape()
    probe.close()
    tuned_shape = {"half": tuned.half, "lanes": tuned.lanes, "rounds": tuned.rounds,
                   "candidates_per_advance": tuned.lanes * (2 * tuned.half + 1) * tuned.rounds}
    plain_tuned, arm_tuned = plain_arm(dev, searches, None, True)
    log(f"batched leg: plain engine (tuned shape {tuned_shape}) {len(searches)} searches in {arm_tuned['wall_s']:.2f} s")
    # the same loop with a short round (half 256, two waves of resident
    # blocks: 9.7e7 candidates an advance), which overshoots a small quota
    # less, and the exact match on the device, as the batch has it
    short = N.EngineConfig(N.SCHEME_PAIRED, SHORT_HALF, 2 * gpu.resident_lanes(dev), 1, 128, 0, 0)
    plain_short, arm_short = plain_arm(dev, searches, short, True)
    log(f"batched leg: plain engine (half {SHORT_HALF}) in {arm_short['wall_s']:.2f} s")

    t0 = time.perf_counter()
    b = B.Batch(dev, **shape, max_half=HALF)
    t_created = time.perf_counter()
    for s in searches:
        b.admit(s.index, s.seed, s.prefixes, s.quota)
    t_admitted = time.perf_counter()
    halves = {s.index: b.status(s.index).half for s in searches}
    steps = launches = 0
    dev_ms = 0.0
    examined = 0
    while b.running():
        b.step()
        steps += 1
        launches += b.last_step_launches()
        dev_ms += b.last_step_ms()
        examined += b.last_step_candidates()
    batched = {s.index: [(h.offset, h.packed) for h in b.results(s.index)] for s in searches}
    b.close()
    batched_wall = time.perf_counter() - t0
    log(f"batched leg: batched engine in {batched_wall:.2f} s, {steps} steps")
    useful = sum(r[-1][0] // 8 for r in batched.values())
    long_ids = [s.index for s in searches if s.expected_candidates() > LONG_SEARCH]
    useful_long = sum(batched[i][-1][0] // 8 for i in long_ids)
    for arm in (arm_tuned, arm_short):
        arm["keys_per_s"] = useful / arm["wall_s"]
    best_plain = min(arm_tuned["wall_s"], arm_short["wall_s"])
    best_name = "tuned" if arm_tuned["wall_s"] <= arm_short["wall_s"] else f"half {SHORT_HALF}"
    best_arm = arm_tuned if best_name == "tuned" else arm_short
    return {
        "workload": "config 4: 64 searches, seeds LE32(j), 1..5000 prefixes (log-uniform) of 4..7 symbols, "
        "quota 1..16" + ("" if cap == float("inf") else "; searches with expected work <= %.0e candidates" % cap),
        "searches": len(searches),
        "searches_in_config": len(all_searches),
        "expected_candidates": sum(s.expected_candidates() for s in searches),
        "candidates_to_quota": useful,
        "results_identical": plain_tuned == batched and plain_short == batched,
        "plain_tuned": {"shape": tuned_shape, "constructor": "og_engine_new(threads = 0), the tuned shape",
                        "match": "device (og_engine_match_on_device)", **arm_tuned},
        "plain_half256": {"shape": {"half": SHORT_HALF, "lanes": short.lanes, "rounds": 1},
                          "constructor": "og_engine_new_config", "match": "device (og_engine_match_on_device)",
                          **arm_short},
        "batched": {"wall_s": batched_wall, "examined": examined, "keys_per_s": useful / batched_wall,
                    "examined_per_s": examined / batched_wall, "device_s": dev_ms / 1e3, "steps": steps,
                    "gpu_launches": launches, "halves": sorted(set(halves.values())),
                    "create_s": t_created - t0, "admit_s": t_admitted - t_created,
                    "long_search_halves": [halves[i] for i in long_ids],
                    "shape": {**shape, "max_half": HALF, "inflight": 2}},
        "speedup_batched_over_plain": best_plain / batched_wall,
        "speedup_against": f"the faster plain arm ({best_name})",
        "speedup_over_plain_tuned": arm_tuned["wall_s"] / batched_wall,
        "speedup_over_plain_half256": arm_short["wall_s"] / batched_wall,
        "long_searches": {
            "count": len(long_ids),
            "candidates_to_quota": useful_long,
            "share_of_work": useful_long / useful,
            "plain_wall_s": best_arm["long_searches_wall_s"],
            "kernel_rate": kernel_rate,
            "bound_note": "no engine examines candidates faster than the single-search kernel at half 2048 "
            "(kernel_rate, the plain line's keys/s): over the faster plain arm a batch is at most its wall / "
            "(all candidates to quota / kernel_rate) faster, and at most its wall / (the long searches' "
            "candidates / kernel_rate) even with the short searches free",
            "speedup_bound": best_plain / (useful / kernel_rate) if kernel_rate else None,
            "speedup_bound_short_free": best_plain / (useful_long / kernel_rate) if kernel_rate else None,
        },
        "unit": "keys/s (candidates up to each search's quota-th hit, wall clock)",
    }


def serving_leg(dev, shape, n, cap_s):
    """Config 5: requests submitted at their Poisson arrival times, served
    until all complete or the wall-clock cap. Time-to-find is completion
    minus arrival; a request still queued or running at the cap has taken at
    least the cap's end minus its arrival, and enters the percentiles with
    that lower bound (a censored value)."""
    from onion_gen_b200 import serve, workloads

    reqs = workloads.config5_requests(n)
    s = serve.Server(dev, **shape)
    t0 = s.now_ns()
    submitted = 0
    sub_ns = {}
    done = {}
    while True:
        now = (s.now_ns() - t0) / 1e9
        while submitted < n and reqs[submitted].arrival <= now:
            r = reqs[submitted]
            s.submit(r.index, r.seed, r.prefixes, r.quota)
            sub_ns[r.index] = s.now_ns()
            submitted += 1
        for d in s.poll():
            done[d.request_id] = d
        if len(done) == n or now > cap_s:
            break
        time.sleep(0.002)
    end_ns = s.now_ns()
    elapsed = (end_ns - t0) / 1e9
    log(f"serving leg: {len(done)} of {submitted} done in {elapsed:.1f} s")
    st = s.stats()
    s.close()
    ok = [d for d in done.values() if d.status == 0]
    failed = [d for d in done.values() if d.status != 0]
    # (seconds, censored): completed exactly; unfinished at least end - arrival
    ttf = [((d.done_ns - d.arrival_ns) / 1e9, False) for d in ok]
    ttf += [((end_ns - sub_ns[r.index]) / 1e9, True) for r in reqs[:submitted] if r.index not in done]
    ttf.sort()

    def q(p):
        if not ttf:
            return None, None
        v, c = ttf[min(len(ttf) - 1, max(0, math.ceil(p * len(ttf)) - 1))]
        return v, c

    p50, c50 = q(0.50)
    p99, c99 = q(0.99)
    return {
        "workload": f"config 5: {n} requests, Poisson arrivals at 50/s (splitmix64(5)), "
        "1..200 prefixes (log-uniform) of 4..7 symbols, quota 1..16",
        "submitted": submitted,
        "completed": len(ok),
        "failed": len(failed),
        "unfinished_at_cap": submitted - len(done),
        "wall_cap_s": cap_s,
        "elapsed_s": elapsed,
        "p50_ttf_s": p50,
        "p50_censored": c50,
        "p99_ttf_s": p99,
        "p99_censored": c99,
        "ttf_note": "percentiles over all submitted requests; a request unfinished at the cap counts with its "
        "elapsed time (cap end - arrival), a lower bound, and a percentile that lands on one is marked censored. "
        "The mix's expected work (2.4e13 candidates, 20 minutes of one GPU) is about 30 times what arrives per "
        "second of capacity, so its longest requests cannot finish within the cap",
        "keys_per_s": st.candidates / elapsed,
        "device_busy": st.device_ms / 1e3 / elapsed,
        "steps": int(st.steps),
    }


def config3_leg(dev, peak, steps=2):
    """Config 3 on its default shape with the exact match on the device: the
    search kernel's keys/s (CUDA events) and roofline fraction, and the same
    candidates end to end through the engine's launch/collect with every
    match copied back and a sample of them re-derived on the host."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    prefixes = workloads.config3_prefixes()
    fs = F.FilterSet.parse_all(prefixes)
    words, bits = fs.index_words()
    seed = workloads.seed(0)
    eng = gpu.Engine(dev, key.start_point(seed), bitmap=words, bitmap_bits=bits,
                     config=N.EngineConfig(N.SCHEME_PAIRED, 0, 0, 0, 128, 0, 0))
    eng.match_on_device(fs)
    shape = eng.shape()
    batch = eng.batch()
    advances = -(-CANDIDATES_PER_STEP // batch)
    eng.advance_matches_raw()  # warm-up
    # the matches cross into the engine's pinned host memory, in og_match's
    # layout, and og_engine_collect_matches_view hands them over there, as a
    # caller in C takes them; only the sampled ones become Python objects
    import ctypes as C

    kernel_ms = 0.0
    matches = checked = 0
    rng = np.random.default_rng(3)
    err = N.errbuf()
    nout = C.c_size_t()
    view = C.c_void_p()
    t0 = time.perf_counter()
    total = steps * advances
    launched = 0
    for i in range(total):
        while launched - i < 2 and launched < total:
            N.check(N.lib.og_engine_launch_matches(eng._h, err, 512), err)
            launched += 1
        N.check(N.lib.og_engine_collect_matches_view(eng._h, C.byref(view), C.byref(nout), err, 512), err)
        kernel_ms += eng.last_kernel_ms()
        m = nout.value
        matches += m
        buf = (N.Match * m).from_address(view.value) if m else []
        for j in rng.choice(m, size=min(64, m), replace=False):
            h = buf[int(j)]
            pk, _ = key.check_hit(seed, int(h.offset), bytes(h.packed))
            if fs.match_address(pk) != int(h.filter):
                raise RuntimeError(f"config 3: match at offset {int(h.offset)} does not confirm on the host")
            checked += 1
    wall = time.perf_counter() - t0
    eng.close()
    n = batch * total
    w = pp_per_candidate(shape.half)
    rate = n / (kernel_ms * 1e-3)
    log(f"config 3 leg: {rate:.4e} keys/s device, {n / wall:.4e} end to end, {matches} matches")
    return {
        "workload": "config 3: seed LE32(0), 10,000 prefixes of 3..8 symbols (splitmix64(3)), "
        f"{bits}-bit index, {steps} steps of 2^32 candidates (rounded up to whole advances), device exact match",
        "shape": {"half": shape.half, "lanes": shape.lanes, "rounds": shape.rounds, "advances_per_step": advances},
        "candidates": n,
        "keys_per_s": rate,
        "roofline_frac": rate * w / peak,
        "per_candidate": w,
        "e2e_keys_per_s": n / wall,
        "matches": matches,
        "match_fraction": matches / n,
        "matches_rederived": checked,
        "e2e_note": "every match crosses to the host in og_match's layout (48 bytes each, 5 % of the "
        "candidates) into the engine's pinned memory, handed over there by og_engine_collect_matches_view, "
        "with 64 of each advance's matches re-derived and confirmed on the host",
        "unit": "keys/s (CUDA events on the search kernel; e2e: wall clock with every match copied back)",
    }


BLOCK_LANES = 128  # lanes a block of the search kernels, which share one inversion


def block_inversion_pp():
    """Partial products a lane spends on its share of the block's one
    inversion: 16 multiplications of its own (two five-step warp scans, the
    other three warps' totals, the last three products) and 1/128 of thread
    0's (three multiplications for the block's product and the inversion,
    254 squarings of 36 products and 11 multiplications)."""
    return 16 * 64 + (14 * 64 + 254 * 36) / BLOCK_LANES


def pp_per_candidate(half):
    """Partial products per candidate of the paired round: 10 + 10 half
    multiplications of 64 and the lane's share of the block's inversion,
    over 2 half + 1 keys."""
    return ((10 + 10 * half) * 64 + block_inversion_pp()) / (2 * half + 1)


def small_case(args):
    """Three advances of one round each: the case the ncu summaries under
    profiles/ are captured on. Half 256 (or --half) keeps the scratch of the
    persistent CTAs near 3.8 GB; the lanes are eight blocks per resident CTA
    (SMs x 5 x 128 x 8), as in production. The kernel is the production one,
    and its DRAM bytes per candidate do not depend on the shape (64 B written
    and read back per candidate)."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    dev = gpu.look()[0]
    half = args.half or 256
    lpt = args.lanes_per_thread
    fs = F.FilterSet.parse_all([workloads.config2_prefix()])
    words, bits = fs.index_words()
    start = key.start_point(workloads.seed(0))
    # eight blocks of lanes per resident CTA (lanes 0: the engine's default waves)
    eng = gpu.Engine(dev, start, bitmap=words, bitmap_bits=bits,
                     config=N.EngineConfig(0, half, 0, 1, 128, 0, 0, lpt))
    lanes = eng.threads()
    for i in range(3):
        o, _ = eng.advance_raw()
        ms = eng.last_kernel_ms()
        print(f"advance {i}: half {half}, {lanes} lanes ({lpt} a thread), {len(o)} survivors, kernel {ms:.3f} ms, "
              f"{eng.batch() / ms * 1e3:.4e} keys/s")


def chain_small_case(args):
    """Three advances of the chain scheme on config 2's search at its default
    shape (n = 1024, four waves of lanes): the case the chain kernel's ncu
    summary is captured on."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    dev = gpu.look()[0]
    fs = F.FilterSet.parse_all([workloads.config2_prefix()])
    words, bits = fs.index_words()
    eng = gpu.Engine(dev, key.start_point(workloads.seed(0)), bitmap=words, bitmap_bits=bits,
                     config=N.EngineConfig(N.SCHEME_CHAIN, args.half, 0, 1, 128, 0, 0))
    for i in range(3):
        o, _ = eng.advance_raw()
        ms = eng.last_kernel_ms()
        print(f"advance {i}: n {eng.shape().half}, {eng.threads()} lanes, {len(o)} survivors, kernel {ms:.3f} ms, "
              f"{eng.batch() / ms * 1e3:.4e} keys/s")


def suffix_small_case(args):
    """Three advances of a suffix search (og_engine_new_filters, forty
    eight-symbol suffixes, half 256, one resident wave): the case the suffix
    match kernel's ncu summary is captured on."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    dev = gpu.look()[0]
    fs = F.FilterSet.parse_all(workloads.suffix_filters(40, 8))
    start = key.start_point(workloads.seed(0))
    lanes = gpu.resident_lanes(dev)
    eng = gpu.Engine(dev, start, filters=fs, config=N.EngineConfig(0, args.half or 256, lanes, 1, 128, 0, 0))
    for i in range(3):
        o, _, _ = eng.advance_matches_raw()
        print(f"advance {i}: {len(o)} matches, search kernel {eng.last_kernel_ms():.3f} ms")


def config3_small_case(args):
    """Three advances of config 3's search (10,000 prefixes of 3..8 symbols,
    a 24-bit index; 5 % of the candidates survive) at its default shape, or
    --half: the case config 3's kernel summaries are captured on."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    dev = gpu.look()[0]
    fs = F.FilterSet.parse_all(workloads.config3_prefixes())
    words, bits = fs.index_words()
    eng = gpu.Engine(dev, key.start_point(workloads.seed(0)), bitmap=words, bitmap_bits=bits,
                     config=N.EngineConfig(N.SCHEME_PAIRED, args.half, 0, 1, 128, 0, 0, args.lanes_per_thread))
    shape = eng.shape()
    for i in range(3):
        o, _ = eng.advance_raw()
        ms = eng.last_kernel_ms()
        print(f"advance {i}: half {shape.half}, {shape.lanes} lanes, {bits}-bit index, {len(o)} survivors, "
              f"kernel {ms:.3f} ms, {eng.batch() / ms * 1e3:.4e} keys/s")


def chain_pp_per_candidate(n):
    """Partial products per candidate of the chain scheme (the config-1
    contract, src/batch.rs:78-122): 7 multiplications for the +8G step, 4 for
    Montgomery's trick and y / Z, and the lane's share of the block's
    inversion per n steps."""
    return (11 * 64 * n + block_inversion_pp()) / n


def chain_leg(dev, peak):
    """The chain scheme (the device restatement of BatchEngine, which config 1
    pins bit for bit) on config 2's search at its default shape (n = 1024,
    four waves of lanes): one warm-up advance, then three timed by CUDA
    events."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    fs = F.FilterSet.parse_all([workloads.config2_prefix()])
    words, bits = fs.index_words()
    eng = gpu.Engine(dev, key.start_point(workloads.seed(0)), bitmap=words, bitmap_bits=bits,
                     config=N.EngineConfig(N.SCHEME_CHAIN, 0, 0, 1, 128, 0, 0))
    shape = eng.shape()
    eng.advance_raw()
    ms = 0.0
    for _ in range(3):
        eng.advance_raw()
        ms += eng.last_kernel_ms()
    rate = 3 * eng.batch() / (ms * 1e-3)
    eng.close()
    w = chain_pp_per_candidate(shape.half)
    log(f"chain leg: {rate:.4e} keys/s at n = {shape.half}, {shape.lanes} lanes")
    return {
        "workload": "chain scheme on config 2's search (seed LE32(0), its 16-bit index), n = %d steps per lane "
        "between inversions, %d lanes" % (shape.half, shape.lanes),
        "keys_per_s": rate,
        "per_candidate": w,
        "roofline_frac": rate * w / peak,
        "unit": "keys/s (CUDA events on the search kernel)",
    }


def suffix_leg(dev, steps, advances):
    """A suffix search through the filter engine (og_engine_new_filters +
    og_engine_advance_matches): the search kernel with the suffix bitmap, the
    device match (full key, sign bit and SHA3-256 checksum recomputed for each
    suffix survivor) and the host's re-derivation of every match."""
    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, workloads

    suffixes = workloads.suffix_filters()
    fs = F.FilterSet.parse_all(suffixes)
    seed = workloads.seed(0)
    eng = gpu.Engine(dev, key.start_point(seed), filters=fs,
                     config=N.EngineConfig(N.SCHEME_PAIRED, HALF, 0, 0, 128, 0, 0))
    eng.advance_matches_raw()
    texts = fs.texts()
    matches = verified = 0
    kernel_ms = 0.0
    t0 = time.perf_counter()
    total = steps * advances
    launched = 0
    for i in range(total):
        while launched - i < 2 and launched < total:
            eng.launch_matches()
            launched += 1
        o, k, f = eng.collect_matches_raw()
        kernel_ms += eng.last_kernel_ms()
        for off, packed, fi in zip(o, k, f):
            pk, _ = key.check_hit(seed, int(off), bytes(packed))
            matches += 1
            verified += fs.match_address(pk) == int(fi) and texts[int(fi)].startswith("suffix:")
    wall = time.perf_counter() - t0
    n = eng.batch() * steps * advances
    eng.close()
    sb = fs.suffix_index_words()[1]
    log(f"suffix leg: {n:.3e} candidates in {wall:.2f} s, {matches} matches")
    return {
        "workload": "suffix search: seed LE32(0), 16 suffixes of 9 symbols (splitmix64(6)), "
        f"suffix bitmap {sb} bits, {steps} steps of {advances} advances",
        "candidates": n,
        "keys_per_s": n / wall,
        "search_kernel_keys_per_s": n / (kernel_ms * 1e-3),
        "matches": matches,
        "matches_verified": verified,
        "expected_matches": n * len(suffixes) * 2.0 ** -37,
        "unit": "keys/s (wall clock, device match and host re-derivation included)",
    }


def batch_small_case(args):
    """Three steps of the batched engine with the first 16 config-4 searches
    admitted (two of them long), at the batched leg's shape except for the
    largest inversion batch: half 256, long searches at up to 512 (the leg
    uses 2048; 512 keeps the scratch near 6 GB for a multi-pass capture), two
    waves of slots, two steps in flight. The case the batched kernels' ncu
    summaries are captured on."""
    from onion_gen_b200 import batch as B
    from onion_gen_b200 import gpu, workloads

    dev = gpu.look()[0]
    half = args.half or SHORT_HALF
    b = B.Batch(dev, half=half, max_half=2 * half)
    for s in workloads.config4_searches()[:16]:
        b.admit(s.index, s.seed, s.prefixes, s.quota)
    print("halves:", sorted(b.status(s.index).half for s in workloads.config4_searches()[:16]))
    for i in range(3):
        b.step()
        ms = b.last_step_ms()
        print(f"step {i}: {b.last_step_candidates()} candidates, {ms:.3f} ms, "
              f"{b.last_step_candidates() / ms * 1e3:.4e} keys/s, running {b.running()}")


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.case == "small":
        small_case(args)
        return
    if args.case == "batch-small":
        batch_small_case(args)
        return
    if args.case == "suffix-small":
        suffix_small_case(args)
        return
    if args.case == "chain-small":
        chain_small_case(args)
        return
    if args.case == "config3-small":
        config3_small_case(args)
        return
    rank, world, local = dist_env()
    import ctypes as C

    import torch

    from onion_gen_b200 import _native as N
    from onion_gen_b200 import filter as F
    from onion_gen_b200 import gpu, key, shard, workloads

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
    # rank r searches its own range of offsets (shard.RANK_SHIFT apart)
    base = shard.rank_start(seed, rank)

    cfg = N.EngineConfig(N.SCHEME_PAIRED, args.half or HALF, 0, 0, 128, 0, 0)
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
    log(f"plain line: {sum(dev_ms):.1f} ms device time over {args.steps} steps")
    total_ms, wall = shard.max_over_ranks([sum(dev_ms), wall])
    keys = batch * advances * args.steps * world
    value = keys / (total_ms * 1e-3)

    # integer-multiply roofline
    imad = C.c_double()
    mulpp = C.c_double()
    err = N.errbuf()
    N.check(N.lib.og_measure_int_peak(dev.ordinal, C.byref(imad), C.byref(mulpp), err, 512), err)
    w = pp_per_candidate(shape.half)
    hbm_peak = None
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except (OSError, KeyError, ValueError):
        hbm_peak = 6650.0  # the pool's earlier measurement, when the driver's file is absent
    achieved = value / world * w
    peak = imad.value / 2.0
    clock_summary = clocks.summary()
    theoretical = (dev.sms * 32 * clock_summary["sm_mhz"] * 1e6) if clock_summary.get("sm_mhz") else None

    # end to end through the C ABI, host buffers, every hit re-derived. As
    # the reference's device worker (src/run.rs:1030-1119) does, one engine
    # serves the whole run: it is created inside the timed region (host
    # precompute, H2D of the start point, tables and bitmap), and every step
    # is `advances` advances with the D2H of their survivors and the host's
    # checks. The clock stops when the last step's hits are verified; the
    # engine's free comes after every result is delivered and is reported
    # beside it (freeing 25 GB of scratch usually takes 0.02 s, but some
    # runs saw 0.2-0.8 s inside cudaFree).
    eng.close()  # the plain line's engine is done; the e2e run makes its own
    e2e = None
    if not args.no_e2e:
        h2d = d2h = 0
        hits = 0
        e2e_steps = args.steps
        barrier()
        t1 = time.perf_counter()
        e = gpu.Engine(dev, base, bitmap=words, bitmap_bits=bits, config=cfg)
        h2d += 128 + words.nbytes + shape.half * 96
        t_created = time.perf_counter()
        total = e2e_steps * advances
        launched = 0
        for i in range(total):
            # two advances in flight: the next one runs while this one's
            # survivors cross back and are checked
            while launched - i < 2 and launched < total:
                e.launch()
                launched += 1
            o, k = e.collect_raw()
            d2h += 16 + 48 * len(o)
            matched = fs.match_many(k)
            for j in np.nonzero(matched >= 0)[0]:
                key.check_hit(seed, shard.global_offset(rank, int(o[j])), bytes(k[j]))
                hits += 1
        t_advanced = time.perf_counter()
        barrier()  # every rank has its results
        e2e_wall = time.perf_counter() - t1
        e.close()
        free_s = time.perf_counter() - t1 - e2e_wall
        e2e = {
            "value": batch * advances * e2e_steps * world / e2e_wall,
            "unit": "keys/s",
            "h2d_bytes_per_step": h2d // e2e_steps,
            "d2h_bytes_per_step": d2h // e2e_steps,
            "steps": e2e_steps,
            "hits_verified": hits,
            "engine_create_s": t_created - t1,
            "timed": "engine creation, then each step's advances with their D2H and the host's checks of every "
            "hit; the engine's free after the last result is engine_free_s, outside",
            "engine_free_s": free_s,
        }
        log(f"e2e: create {t_created - t1:.3f} s, {e2e_steps} steps {t_advanced - t_created:.3f} s, "
            f"free {free_s:.3f} s")

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
                "workload": plain_workload(prefix),
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
                "traffic": TRAFFIC_PER_CANDIDATE * batch,
                "traffic_unit": "DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum on the "
                "small case, 128.6 B a candidate, scaled to this launch's candidates)",
                "per_candidate": w,
                "peak_source": "measured: og_measure_int_peak mad.lo.u32 issue rate / 2 (lo+hi per product)",
                "peak_theoretical": theoretical,
                "peak_theoretical_source": "SMs x 32 wide 32x32->64 multiply-adds a clock (fmaheavy) x the median "
                "SM clock sampled during the timed steps",
                "frac_of_theoretical": achieved / theoretical if theoretical else None,
                "fe_mul_pp_per_s": mulpp.value,
                "hbm": {
                    "achieved": value / world * ALGORITHMIC_BYTES_PER_CANDIDATE / 1e9,
                    "peak": hbm_peak,
                    "unit": "GB/s",
                    "frac": value / world * ALGORITHMIC_BYTES_PER_CANDIDATE / 1e9 / hbm_peak if hbm_peak else None,
                    "note": "the Montgomery scratch: not the bound",
                },
            },
            "clocks": clock_summary,
        }
        if e2e:
            line["e2e"] = e2e
        if world > 1:
            # the CPU baseline and the single-GPU legs (suffix, batched,
            # serving) describe one GPU and its host: they run at N = 1 only,
            # so that N GPUs are not held for them
            line["legs"] = "the CPU baseline and the suffix, batched and serving legs run at N = 1 only"
            print(json.dumps(line), flush=True)
            if pg:
                pg.destroy_process_group()
            return
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        if args.suite == "default":
            line["chain"] = chain_leg(dev, peak)
        if args.suite in ("default", "suffix"):
            line["suffix"] = suffix_leg(dev, 2 if args.suite == "default" else args.steps, advances)
        if args.suite in ("default", "config3"):
            line["config3"] = config3_leg(dev, peak)
        if args.suite in ("default", "batched", "serving"):
            shape, line["batch_shape"] = batch_shape(dev)
        if args.suite in ("default", "batched"):
            line["batched"] = batched_leg(dev, shape, args.batched_cap, value)
        if args.suite in ("default", "serving"):
            line["serving"] = serving_leg(dev, shape, args.serving_requests, args.serving_cap)
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
