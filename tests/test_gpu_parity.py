"""Sequential parity of the CUDA allocator with the oracle (and so with the
reference): one GPU thread replays every trace of tests/golden/traces.py; every
result (size class, chunk, page) and every counter must be identical."""
import numpy as np
import pytest

import oracle
import ouroboros_b200 as ob
from tests.golden import traces

pytestmark = pytest.mark.gpu

STATE_NAMES = ["next_free_chunk", "reuse0.count", "reuse0.front", "reuse0.back", "reuse1.count", "reuse1.front",
               "reuse1.back"] + [f"class{c}.{f}" for c in range(12) for f in (
                   "count", "expected", "reserved", "front", "back", "entries", "front_ptr", "back_ptr", "old_ptr",
                   "old_count", "va_digest", "ppc")]


def _diff(a, b):
    idx = np.nonzero(a != b)[0]
    return [(STATE_NAMES[i], int(a[i]), int(b[i])) for i in idx[:8]]


@pytest.mark.parametrize("v", ob.VARIANTS)
def test_init_state_matches_oracle(v):
    with ob.Ouroboros(v, traces.HEAP_BYTES) as heap:
        st = heap.state()
        info = heap.info()
    o = oracle.Oracle(v, traces.HEAP_BYTES)
    assert info["max_chunks"] == oracle.layout(v, traces.HEAP_BYTES)["max_chunks"]
    assert np.array_equal(st, o.state()), _diff(st, o.state())


@pytest.mark.parametrize("name", list(traces.TRACES))
@pytest.mark.parametrize("v", ob.VARIANTS)
def test_trace_matches_oracle(v, name):
    ops, tid, bid = traces.build(name)
    with ob.Ouroboros(v, traces.heap_bytes(name)) as heap:
        got = heap.trace(ops, tid, bid)
        st = heap.state()
        flags = heap.status()["flags"]
    o = oracle.Oracle(v, traces.heap_bytes(name), tid, bid)
    want, _ = o.run_trace(ops)
    assert flags == 0
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"op {bad[0]}: got {oracle.decode(int(got[bad[0]]))} oracle {oracle.decode(int(want[bad[0]]))}"
    ost = o.state()
    assert np.array_equal(st, ost), _diff(st, ost)


@pytest.mark.parametrize("v", ob.VARIANTS)
def test_initial_chunk_entry_points_match_oracle(v):
    # The host entry points (ouro_allocate_chunk, ouro_enqueue_initial_chunk)
    # on a fresh heap, then a sequential trace: its mallocs take the initial
    # pages first, in the oracle's order, and the counters agree.
    with ob.Ouroboros(v, traces.HEAP_BYTES) as heap:
        c = heap.allocate_chunk()
        heap.enqueue_initial_chunk(3, c, 40)    # 128 B pages (64 a chunk): 24 held by the caller, 40 free
        ops = np.array([0, 128] * 130, dtype=np.uint32)
        got = heap.trace(ops)
        st = heap.state()
        with pytest.raises(ob.OuroError):
            heap.enqueue_initial_chunk(3, c, 65)    # more pages than the chunk has
    o = oracle.Oracle(v, traces.HEAP_BYTES)
    oc = o.run_trace(np.array([2, 0, 3, (0 << 14) | (40 << 4) | 3], dtype=np.uint32))[0][0]
    assert int(oc) == c
    want, _ = o.run_trace(ops)
    assert np.array_equal(got, want)
    # the first 40 requests take the 40 free pages of the initial chunk (page
    # order for page queues, the bitmask search order for chunk queues)
    first = [oracle.decode(int(r)) for r in got[:40]]
    assert all(chunk == c and page >= 24 for _, chunk, page in first)
    assert len({page for _, _, page in first}) == 40
    assert np.array_equal(st, o.state()), _diff(st, o.state())
