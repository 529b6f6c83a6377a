"""Failure detection without a GPU fault: a bounded device wait on a barrier
that nothing completes gives up, is reported as ETIMEOUT, and the context
keeps working; a failed request does not stop the server (see
test_gpu_server.py) and bad inputs are rejected before any launch."""
import time

import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(gpu_ctx):
    t0 = time.time()
    limit_us = 50_000
    status, waited_ns = gpu_ctx.selftest_bounded_wait(limit_us)
    assert status == cuapss.ETIMEOUT
    # the deadline is device time: it waited at least the limit, and gave up
    # soon after it (one try-wait suspends for at most 20 us)
    assert waited_ns >= limit_us * 1000
    assert waited_ns <= 3 * limit_us * 1000
    assert time.time() - t0 < 30.0
    # twice in a row, then real work on the same context
    status, waited_ns = gpu_ctx.selftest_bounded_wait(1)
    assert status == cuapss.ETIMEOUT and 1000 <= waited_ns < 10_000_000
    x = synth.generate("plain_20k", n=1500)
    i, j, s = gpu_ctx.run(x, 0.7)
    wi, wj, ws = oracle.apss(x, 0.7)
    assert np.array_equal(i, wi) and np.array_equal(j, wj)


def test_bounded_wait_limit_of_the_tile_kernels(gpu_ctx):
    # the full 2 s deadline the tile kernels use
    status, waited_ns = gpu_ctx.selftest_bounded_wait(2_000_000)
    assert status == cuapss.ETIMEOUT
    assert 2.0e9 <= waited_ns <= 2.5e9


def test_bounded_wait_rejects_bad_limits(gpu_ctx):
    assert gpu_ctx.selftest_bounded_wait(0)[0] == cuapss.EINVAL
    assert gpu_ctx.selftest_bounded_wait(2_000_001)[0] == cuapss.EINVAL
