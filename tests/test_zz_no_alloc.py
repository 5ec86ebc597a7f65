"""og_search_noalloc, the search entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc themselves or have the library
call it — code running inside another framework's memory pool, callers that
must not trigger the device synchronisation an allocation or a free can
cause, processes that reserve all device memory up front. They hand in device
buffers they already own; the library's scratch is a fixed device array.

Checked on a B200 (-m gpu) through the C ABI against og_engine_advance on a
fresh engine of the same shape: the same survivors, bit for bit, on two calls
in a row (a filtered one, then one that keeps every candidate), then the
first again; and a call made behind a finite spin kernel on the same stream
returns before that kernel ends (it copies nothing from host memory, so it
does not wait for queued work). This file is collected last, so a run that stops at the first
failure has run every other test before it.
"""
import time

import numpy as np
import pytest
import torch

from onion_gen_b200 import _native as N
from onion_gen_b200 import filter as F
from onion_gen_b200 import gpu, key, workloads

pytestmark = pytest.mark.gpu

LANES, HALF, ROUNDS = 1024, 64, 2
SLOTS = 2 * HALF + 1


def with_engine(device, start, words, bits, dump):
    cfg = N.EngineConfig(N.SCHEME_PAIRED, HALF, LANES, ROUNDS, 128, 1 if dump else 0, 0)
    eng = gpu.Engine(device, start, bitmap=None if dump else words, bitmap_bits=bits, config=cfg)
    offsets, packed = eng.advance_raw()
    eng.close()
    return sorted(zip(offsets.tolist(), (bytes(p) for p in packed)))


def without_allocation(device, start, d_bitmap, bits, cap, stream=None):
    # the caller's own device buffers: survivor records and their counter
    d_hits = torch.zeros(cap * 12, dtype=torch.int32, device=f"cuda:{device.ordinal}")
    d_count = torch.full((1,), 12345, dtype=torch.int32, device=f"cuda:{device.ordinal}")
    err = N.errbuf()
    rc = N.lib.og_search_noalloc(
        device.ordinal, start, LANES, HALF, ROUNDS, d_bitmap, bits, d_hits.data_ptr(), cap, d_count.data_ptr(), stream,
        err, 512,
    )
    N.check(rc, err)
    torch.cuda.synchronize()
    n = int(d_count.item())
    assert 0 < n <= cap
    recs = d_hits[: n * 12].cpu().numpy().view(np.uint32).reshape(n, 12)
    out = []
    for rec in recs:
        lane, step = int(rec[0]), int(rec[1])
        w = (step // SLOTS) * LANES + lane
        out.append((8 * (w * SLOTS + 1 + step % SLOTS), rec[4:12].astype("<u4").tobytes()))
    return sorted(out)


def test_no_allocation_entry_point_matches_the_engine(device):
    fs = F.FilterSet.parse_all(["ab", "q7"])
    words, bits = fs.index_words()
    d_bitmap = torch.from_numpy(words.view(np.int64)).to(f"cuda:{device.ordinal}")
    start_a = key.start_point(workloads.seed(3))
    start_b = key.start_point(workloads.seed(4))
    n = LANES * ROUNDS * SLOTS

    first = without_allocation(device, start_a, d_bitmap.data_ptr(), bits, cap=n)
    assert first == with_engine(device, start_a, words, bits, dump=False)
    assert len(first) > 100

    second = without_allocation(device, start_b, None, 0, cap=n)
    assert second == with_engine(device, start_b, words, bits, dump=True)
    assert [o for o, _ in second] == [8 * (i + 1) for i in range(n)]

    again = without_allocation(device, start_a, d_bitmap.data_ptr(), bits, cap=n)
    assert again == first


def test_no_allocation_entry_point_refuses_sizes_beyond_its_array(device):
    start = key.start_point(workloads.seed(3))
    err = N.errbuf()
    d_hits = torch.zeros(12, dtype=torch.int32, device=f"cuda:{device.ordinal}")
    d_count = torch.zeros(1, dtype=torch.int32, device=f"cuda:{device.ordinal}")
    # 65536 lanes at half 256 need about 2.2 GB of scratch: refused before any device work
    rc = N.lib.og_search_noalloc(device.ordinal, start, 65536, 256, 1, None, 0, d_hits.data_ptr(), 1,
                                 d_count.data_ptr(), None, err, 512)
    assert N.STATUS[rc] == "OG_E_CAPACITY"
    assert b"fixed array" in err.value


def test_no_allocation_entry_point_returns_without_waiting_for_queued_work(device):
    fs = F.FilterSet.parse_all(["ab", "q7"])
    words, bits = fs.index_words()
    dev = f"cuda:{device.ordinal}"
    d_bitmap = torch.from_numpy(words.view(np.int64)).to(dev)
    start = key.start_point(workloads.seed(3))
    n = LANES * ROUNDS * SLOTS
    want = without_allocation(device, start, d_bitmap.data_ptr(), bits, cap=n)  # the device's first call done
    stream = torch.cuda.Stream(device=dev)
    d_hits = torch.zeros(n * 12, dtype=torch.int32, device=dev)
    d_count = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        torch.cuda._sleep(1_000_000_000)  # a finite spin of about half a second at B200 clocks
    err = N.errbuf()
    t0 = time.perf_counter()
    rc = N.lib.og_search_noalloc(device.ordinal, start, LANES, HALF, ROUNDS, d_bitmap.data_ptr(), bits,
                                 d_hits.data_ptr(), n, d_count.data_ptr(), stream.cuda_stream, err, 512)
    returned_s = time.perf_counter() - t0
    still_queued = not stream.query()
    N.check(rc, err)
    stream.synchronize()
    assert still_queued, "the spin kernel had ended before the call returned"
    assert returned_s < 0.1
    m = int(d_count.item())
    recs = d_hits[: m * 12].cpu().numpy().view(np.uint32).reshape(m, 12)
    got = sorted((8 * (((int(r[1]) // SLOTS) * LANES + int(r[0])) * SLOTS + 1 + int(r[1]) % SLOTS),
                  r[4:12].astype("<u4").tobytes()) for r in recs)
    assert got == want
