"""The C oracle against the reference's own outputs (CPU only).

tests/golden/trace_<variant>.npz hold what the reference allocator, compiled for
sm_100a, returned when one GPU thread replayed each trace of traces.py on a
fresh heap of 1 GiB (4 GiB for the large trace; generator:
tests/golden/make_golden.py).  The oracle must
reproduce every byte offset and every counter bit-exactly.
"""
import os

import numpy as np
import pytest

import oracle
from tests.golden import traces
from tests.golden.make_golden import NOT_RUN, offsets_digest, ops_digest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(v):
    return np.load(os.path.join(GOLDEN, f"trace_{v}.npz"))


@pytest.mark.parametrize("v", oracle.VARIANTS)
def test_layout_and_init_state(v):
    g = _golden(v)
    lay = oracle.layout(v, traces.HEAP_BYTES)
    assert lay["max_chunks"] == int(g["meta"][0])
    assert lay["allocation_bytes"] == int(g["meta"][1])
    o = oracle.Oracle(v, traces.HEAP_BYTES)
    assert np.array_equal(o.state(), g["init_state"])


@pytest.mark.parametrize("name", list(traces.TRACES))
@pytest.mark.parametrize("v", oracle.VARIANTS)
def test_trace_bit_exact(v, name):
    if (v, name) in NOT_RUN:
        pytest.skip("the reference's VAC code is not run at this scale (it faulted under concurrency)")
    g = _golden(v)
    ops, tid, bid = traces.build(name)
    assert bytes(g[f"{name}_ops_sha256"]).hex() == ops_digest(ops), "trace generator drifted from the fixture"
    o = oracle.Oracle(v, traces.heap_bytes(name), tid, bid)
    res, off = o.run_trace(ops)
    if name in traces.DIGEST_ONLY:
        assert offsets_digest(off) == bytes(g[f"{name}_off_sha256"]), "offsets differ from the reference's"
    else:
        gold = g[f"{name}_off"]
        bad = np.nonzero(off != gold)[0]
        assert bad.size == 0, f"first mismatch at op {bad[0]}: oracle {off[bad[0]]} reference {gold[bad[0]]}"
    st = o.state()
    sbad = np.nonzero(st != g[f"{name}_state"])[0]
    assert sbad.size == 0, f"state words differ: {sbad.tolist()}"


def test_layout_reference_points():
    # maxChunks quoted for the reference at 1/4/8/16/32 GiB (host probe of the
    # reference types): P/C, VA, VL
    want = {"P": [80596, 467763, 983985, 2016429, 4081317],
            "VAP": [128897, 516064, 1032286, 2064730, 4129618],
            "VLP": [128992, 516159, 1032381, 2064825, 4129713]}
    for v, row in want.items():
        got = [oracle.layout(v, g << 30)["max_chunks"] for g in (1, 4, 8, 16, 32)]
        assert got == row


def test_oracle_rejects_reference_ub():
    # A heap with a handful of chunks: the reference would run past maxChunks
    # (callers ignore allocateChunk's false); the oracle reports it instead.
    heap = oracle.layout("VAP", 1 << 30)["total_required"] + 20 * 8320
    o = oracle.Oracle("VAP", heap)
    with pytest.raises(oracle.OracleError):
        for _ in range(100):
            o.malloc(8192)
