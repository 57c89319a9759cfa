"""CPU checks of the C ABI: the library builds, loads and exports every symbol
that include/ouroboros_b200.h declares (no device calls)."""
import ctypes
import os
import re

import ouroboros_b200 as ob
from ouroboros_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "ouroboros_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|const char\*)\s+(ouro_\w+)\(", hdr, re.M)))


def test_library_builds_and_exports_header():
    path = build.build()
    lib = ctypes.CDLL(path)
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), f"{name} missing from {path}"
    assert sorted(ob.EXPORTS) == declared


def test_status_strings_and_bad_arguments():
    lib = ob.lib()
    assert lib.ouro_status_string(0) == b"ok"
    out = ctypes.c_void_p()
    assert lib.ouro_create(7, 1 << 30, ctypes.byref(out)) == 1          # unknown variant
    assert lib.ouro_create(0, 1 << 20, ctypes.byref(out)) == 1          # below the queue region
    assert lib.ouro_destroy(None) == 1


def test_size_classes_match_oracle_encoding():
    # the class of a request size, as the device code computes it, against the reference rule
    import oracle
    o = oracle.Oracle("P", 1 << 30)
    for size in (0, 1, 15, 16, 17, 31, 32, 33, 100, 4096, 4097, 8192, 8193, 16384, 16385, 32768):
        res, _ = o.malloc(size)
        cls = (res >> 32) & 0xFF
        inst, q = divmod(cls, 16)
        ps = (16 << q) if inst == 0 else (16384 << q)
        assert size <= ps and (size <= 16 if q == 0 and inst == 0 else size > ps // 2 or (inst == 1 and q == 0))


def test_config_defaults_and_refusals_without_a_device():
    # the defaults are the reference's compile-time parameters (include/Parameters.h:9-18)
    c = ob.default_config().as_dict()
    assert c == {"chunk_bytes": 8192, "page_queue_entries": 1 << 23, "virtual_queue_entries": 16384, "agg_width": 32}
    out = ctypes.c_void_p()
    for bad in ({"chunk_bytes": 4096}, {"page_queue_entries": 3 << 16}, {"page_queue_entries": 1 << 24},
                {"virtual_queue_entries": 16}, {"agg_width": 3}, {"agg_width": 0}):
        cfg = ob.default_config(**bad)
        assert ob.lib().ouro_create_config(0, 1 << 30, ctypes.byref(cfg), ctypes.byref(out)) == 1, bad
    assert ob.lib().ouro_config_default(None) == 1


def test_host_buffer_calls_refuse_bad_arguments_without_a_device():
    # argument checks come before any CUDA call: a missing heap is refused
    # (the GPU tests cover the other refusals on a real heap)
    lib = ob.lib()
    buf = (ctypes.c_uint64 * 4)()
    assert lib.ouro_alloc_host(None, 4, 64, None, buf, None, 256, 0, None) == 1
    assert lib.ouro_free_host(None, 4, buf, 256, 0, None) == 1
    assert lib.ouro_host_reserve(None, 4) == 1
