"""The same concurrent workload through the reference's own allocator (its
sm_100a build, oracle/_ref) and through this build: 2^16 threads each
allocating one fixed size, a seeded pattern written and verified through every
pointer, then all freed.  Addresses are nondeterministic in both, so what is
compared is what both must agree on: no null result and no corrupted word in
either, and the pages each class owns afterwards.  This build creates exactly
the chunks the burst needs (ceil(requests / pages per chunk)); the reference
can only create as many or more.

The reference runs only where its code has run cleanly here: its VAC and VLC
code faulted on other workloads and is not run again."""
import numpy as np
import pytest
import torch

import oracle
import ouroboros_b200 as ob

pytestmark = pytest.mark.gpu

GiB = 1 << 30
SEED = 0x5EED1234


def _ref_round(v, n, size):
    ref = oracle.RefDriver(v, GiB)
    try:
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        ref.alloc(n, size, ptrs.data_ptr())
        ref.sanitize(n, size, ptrs.data_ptr(), cnt.data_ptr())
        oracle.ref_write(ptrs.data_ptr(), n, size, SEED)
        oracle.ref_verify(ptrs.data_ptr(), n, size, SEED, cnt.data_ptr())
        ref.free(n, ptrs.data_ptr())
        torch.cuda.synchronize()
        return cnt.tolist(), ref.state()
    finally:
        ref.close()


def _our_round(v, n, size):
    with ob.Ouroboros(v, GiB) as heap:
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        heap.alloc(ptrs, n, size)
        ob.write_pattern(ptrs, n, size, SEED)
        ob.verify_pattern(ptrs, n, cnt, size, SEED)
        heap.free(ptrs, n)
        torch.cuda.synchronize()
        assert heap.status()["flags"] == 0
        return cnt.tolist(), heap.state()


@pytest.mark.skipif(not oracle.ref_available(), reason="the reference's sm_100a build is not present")
@pytest.mark.parametrize("size", [16, 64, 1024])
@pytest.mark.parametrize("v", ["P", "C", "VAP", "VLP"])
def test_concurrent_round_against_the_reference(v, size):
    n = 1 << 16
    ref_cnt, ref_state = _ref_round(v, n, size)
    our_cnt, our_state = _our_round(v, n, size)
    assert ref_cnt == [0, 0] and our_cnt == [0, 0], (ref_cnt, our_cnt)
    q = max(int(np.ceil(np.log2(size))) - 4, 0)
    ppc = 512 >> q
    need = -(-n // ppc) * ppc   # pages of the chunks the burst needs
    # word 7 + 12 q: the class's semaphore count, at quiescence its free pages
    ours = int(np.int64(our_state[7 + 12 * q]))
    theirs = int(np.int64(ref_state[7 + 12 * q]))
    assert ours == need, (ours, need)
    assert theirs >= need, (theirs, need)
