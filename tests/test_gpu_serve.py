"""The serving loop on a B200 (-m gpu): requests arriving while others run
are admitted, complete with the same result as alone, and carry consistent
time stamps; a request that cannot run completes with its error status."""
import time

import pytest

from onion_gen_b200 import _native as N
from onion_gen_b200 import batch as B
from onion_gen_b200 import serve, workloads

pytestmark = pytest.mark.gpu

SMALL = dict(half=64, slots=128 * 64)


def requests():
    r = workloads.SplitMix64(505)
    out = []
    for i in range(12):
        n = 1 + r.next() % 40
        out.append((1000 + i, [r.prefix(3, 4) for _ in range(n)], 1 + r.next() % 6))
    return out


def alone(device, rid, prefixes, quota):
    b = B.Batch(device, **SMALL)
    b.admit(rid, workloads.seed(rid), prefixes, quota)
    while b.running():
        b.step()
    res = [(h.offset, h.packed) for h in b.results(rid)]
    b.close()
    return res


def test_serving_results_equal_alone(device):
    reqs = requests()
    with serve.Server(device, **SMALL) as s:
        for rid, prefixes, quota in reqs[:6]:
            s.submit(rid, workloads.seed(rid), prefixes, quota)
        time.sleep(0.05)
        for rid, prefixes, quota in reqs[6:]:
            s.submit(rid, workloads.seed(rid), prefixes, quota)
        s.submit(77, workloads.seed(77), ["a0"], 1)
        done = {}
        deadline = time.time() + 120
        while len(done) < len(reqs) + 1 and time.time() < deadline:
            for d in s.poll():
                done[d.request_id] = d
            time.sleep(0.01)
        assert len(done) == len(reqs) + 1
        assert N.STATUS[done[77].status] == "OG_E_FILTER"
        results = {rid: [(h.offset, h.packed) for h in s.results(rid)] for rid, _, _ in reqs}
        st = s.stats()
        assert st.completed == len(reqs) + 1 and st.steps > 0 and st.running == 0 and st.queued == 0
    for rid, prefixes, quota in reqs:
        d = done[rid]
        assert d.status == 0 and d.hits == quota
        assert d.arrival_ns <= d.admit_ns <= d.done_ns
        assert results[rid] == alone(device, rid, prefixes, quota), rid
