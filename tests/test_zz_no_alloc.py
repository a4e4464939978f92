"""sc_exclusive_scan_u32_noalloc, the allocation-free scan, through the C ABI.

It exists for callers that cannot allocate device memory (a host engine that
owns every device allocation through its own pool, or a latency-critical path
that cannot afford cudaMalloc's implicit synchronisation); its scratch is a
fixed device array inside the library.  Its results must equal the allocating
scan's, call after call, since the shared scratch keeps the previous call's
contents.  This file is collected last so a stop-at-first-failure run has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 26


def _scan(ctx, fn_name, x):
    from nanotracer_b200._lib import check, lib
    buf = ctx.storage_buffer("scan", x)
    tot = ctx.storage_buffer_zeroed("total", 8)
    f = getattr(lib(), fn_name)
    check(f(ctx.handle, buf.cptr, C.c_uint64(len(x)), tot.cptr), ctx.handle)
    return buf.readback(np.uint32), int(tot.readback(np.uint64)[0])


def _bind():
    from nanotracer_b200._lib import lib
    L = lib()
    f = L.sc_exclusive_scan_u32_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
    return L


def test_noalloc_scan_matches_allocating_scan_on_consecutive_calls(ctx):
    _bind()
    rng = np.random.default_rng(99)
    # a large call followed by a smaller one: the second reuses scratch the
    # first left behind, so the clearing of the shared array is exercised
    for n in (5_000_011, 70_001, 5_000_011, 1):
        x = rng.integers(0, 64, n).astype(np.uint32)
        want, want_total = _scan(ctx, "sc_exclusive_scan_u32", x)
        got, got_total = _scan(ctx, "sc_exclusive_scan_u32_noalloc", x)
        assert np.array_equal(got, want) and got_total == want_total
        ref = np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]).astype(np.uint32)
        assert np.array_equal(got, ref)


def test_noalloc_scan_rejects_sizes_beyond_its_scratch(ctx):
    from nanotracer_b200._lib import lib
    _bind()
    x = np.arange(8, dtype=np.uint32)
    buf = ctx.storage_buffer("scan", x)
    st = lib().sc_exclusive_scan_u32_noalloc(ctx.handle, buf.cptr, C.c_uint64(MAX_N + 1), None)
    assert st == 1  # SC_ERR_INVALID_ARG
    assert b"SC_NOALLOC_SCAN_MAX_N" in lib().sc_last_error(ctx.handle)
    assert np.array_equal(buf.readback(np.uint32), x)  # data untouched


def test_noalloc_scan_after_a_timed_out_wait(ctx):
    """A look-back wait that gave up (the failure self-test) leaves the
    context usable; the next allocation-free scan clears the scratch it uses
    and matches the allocating scan."""
    from nanotracer_b200._lib import lib
    _bind()
    assert lib().sc_selftest_wait_timeout(ctx.handle) == 5  # SC_ERR_TIMEOUT
    x = np.random.default_rng(7).integers(0, 1000, 3_000_017).astype(np.uint32)
    want, want_total = _scan(ctx, "sc_exclusive_scan_u32", x)
    got, got_total = _scan(ctx, "sc_exclusive_scan_u32_noalloc", x)
    assert np.array_equal(got, want) and got_total == want_total
