"""GPU parity of the mixed-precision path (BF16 head on tcgen05 tensor
cores, FP32 tail, FP64 rescore of the error band) against the FP64 oracle:
the pair set must be identical and reported similarities within 1e-6."""
import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

from tests.test_gpu_parity import SIM_TOL, _check_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed_ctx():
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    with cuapss.Context(precision=cuapss.PREC_MIXED) as c:
        yield c


def test_mixed_small(mixed_ctx):
    x = synth.generate("plain_20k", n=300)
    _check_pairs(mixed_ctx.run(x, 0.7), oracle.apss(x, 0.7))


@pytest.mark.parametrize("t", [0.9, 0.7, 0.5])
def test_mixed_plain_20k(mixed_ctx, t):
    x = synth.generate("plain_20k")
    got = mixed_ctx.run(x, t)
    _check_pairs(got, oracle.apss(x, t))
    st = mixed_ctx.last_stats
    assert st["candidates"] >= st["pairs"]


@pytest.mark.parametrize("p", [64, 128, 256, 512, 1024])
def test_mixed_head_widths(p):
    x = synth.generate("batch_instance", n=3000, seed=5)
    with cuapss.Context(precision=cuapss.PREC_MIXED, head_width=p) as c:
        got = c.run(x, 0.6)
        assert c.last_stats["head_width"] == p
    _check_pairs(got, oracle.apss(x, 0.6))


def test_mixed_edge_sizes(mixed_ctx):
    full = synth.generate("plain_20k", n=700)
    for n in (0, 1, 2, 127, 128, 129, 300, 700):
        x = full.rows(0, n)
        _check_pairs(mixed_ctx.run(x, 0.5), oracle.apss(x, 0.5))


def test_mixed_cross_join(mixed_ctx):
    x = synth.generate("plain_20k", n=9000)
    a, b = x.rows(0, 3000), x.rows(3000, 9000)
    _check_pairs(mixed_ctx.join(a, b, 0.6), oracle.join(a, b, 0.6))


@pytest.mark.parametrize("n", [3000, 3001 + 128, 5000])
def test_mixed_two_block_mma_tiles(n):
    # a head as wide as d leaves no tail: the plan is head-bound, so the
    # tiles are MMAs of N = 256 over two J blocks (and N = 128 for a unit's
    # last block when its J range has an odd length); self- and cross-join
    x = synth.generate("plain_20k", n=n + 4000)
    d64 = (x.d + 63) // 64 * 64
    a, b = x.rows(0, n), x.rows(n, n + 4000)
    with cuapss.Context(precision=cuapss.PREC_MIXED, head_width=d64) as c:
        _check_pairs(c.run(a, 0.6), oracle.apss(a, 0.6))
        assert c.last_stats["head_width"] == d64
        _check_pairs(c.join(a, b, 0.6), oracle.join(a, b, 0.6))


def test_mixed_matches_fp32_path():
    x = synth.generate("plain_800k", n=30000)
    with cuapss.Context(precision=cuapss.PREC_MIXED) as m, cuapss.Context() as f:
        a = m.run(x, 0.6, capacity=1 << 20)
        b = f.run(x, 0.6, capacity=1 << 20)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.max(np.abs(a[2] - b[2])) <= 2 * SIM_TOL


def test_mixed_known_answers(mixed_ctx):
    v, w = np.float32(0.6), np.float32(0.8)
    rows = [[(1, v), (5, w)], [(1, v), (5, w)], [(2, np.float32(1.0))], [(1, w), (5, v)],
            [(5, np.float32(1.0))]]
    rp, col, val = [0], [], []
    for r in rows:
        for c_, x_ in r:
            col.append(c_)
            val.append(x_)
        rp.append(len(col))
    x = synth.Csr(np.array(rp), np.array(col, np.int32), np.array(val, np.float32), 8)
    for t in (0.5, float(w), float(np.nextafter(w, np.float32(2))), 1.0):
        _check_pairs(mixed_ctx.run(x, t), oracle.apss(x, t))
