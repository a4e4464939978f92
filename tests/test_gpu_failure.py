"""Failure detection on the device without a fault: a bounded look-back wait
that nothing will ever satisfy gives up, the call reports SC_ERR_TIMEOUT, and
the context keeps working."""
import time

import numpy as np
import pytest

from nanotracer_b200._lib import lib

pytestmark = pytest.mark.gpu

SC_ERR_TIMEOUT = 5


def test_bounded_wait_times_out_and_context_survives(ctx):
    from tests.test_gpu_raster import _sort_gpu
    t0 = time.time()
    st = lib().sc_selftest_wait_timeout(ctx.handle)
    dt = time.time() - t0
    assert st == SC_ERR_TIMEOUT, st
    assert dt < 60
    # the error word was read and cleared; the next call works
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 20, 50_000, dtype=np.uint32)
    vals = np.arange(50_000, dtype=np.uint32)
    k, v = _sort_gpu(ctx, keys, vals, 20, 4)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])
