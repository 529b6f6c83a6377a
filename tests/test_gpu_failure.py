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
    status, polls = gpu_ctx.selftest_bounded_wait(200)
    assert status == cuapss.ETIMEOUT
    assert polls == 200
    assert time.time() - t0 < 30.0
    # twice in a row, then real work on the same context
    assert gpu_ctx.selftest_bounded_wait(1)[0] == cuapss.ETIMEOUT
    x = synth.generate("plain_20k", n=1500)
    i, j, s = gpu_ctx.run(x, 0.7)
    wi, wj, ws = oracle.apss(x, 0.7)
    assert np.array_equal(i, wi) and np.array_equal(j, wj)


def test_bounded_wait_rejects_bad_limits(gpu_ctx):
    assert gpu_ctx.selftest_bounded_wait(0)[0] == cuapss.EINVAL
    assert gpu_ctx.selftest_bounded_wait(10**7)[0] == cuapss.EINVAL
