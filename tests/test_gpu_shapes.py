"""GPU parity on the benchmark workloads' real shapes, through the C ABI,
against the FP64 oracle.

* the n = d = 1M mixed-precision workload's distribution (d = 1,000,000,
  Zipf 1.2, rows up to 5,000 entries) at 40,000 rows, both precisions, the
  library's head width and the named 4,096, t in {0.5, 0.7, 0.8};
* the serving workload's index shape (d = 2^20) queried with per-row
  thresholds;
* the n = 800k plain workload's distribution at 60,000 rows, t in {0.5, 0.9};
* the tail-feature key range at its edge (d - p = 2^20 - 2, every feature
  present, so the tail ranks reach the top of the range) and one past it
  (EINVAL);
* blocks whose tails exceed the tile kernels' staging capacity (chunked
  staging) next to blocks that fit.

The reference itself caps feature ids at max_dim = 198,456
(similarity_search.cu:17); these ranges go past it.

Oracle comparisons at 40k-60k rows use sampled query rows (oracle.rows):
every emitted pair that touches a sampled row must be an oracle pair and
vice versa, similarities within 1e-6 of FP64. Size-independent properties
(sorted, unique, i < j, every emitted pair's FP64 value >= t) hold on the
whole output."""
import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6


def _check_pairs(got, want, tol=SIM_TOL):
    gi, gj, gs = got
    wi, wj, ws = want
    assert len(gi) == len(wi), f"pair count {len(gi)} != oracle {len(wi)}"
    assert np.array_equal(gi, wi) and np.array_equal(gj, wj)
    if len(gs):
        err = np.max(np.abs(gs.astype(np.float64) - ws))
        assert err <= tol, f"max |sim - fp64| = {err}"


def _sampled_check(x, got, t, rows, want_low):
    """got: the full self-join at t; want_low: oracle.rows at some t' <= t."""
    gi, gj, gs = got
    assert np.all(gi < gj)
    key = gi.astype(np.int64) * x.n + gj
    assert np.all(np.diff(key) > 0), "output not sorted / not unique"
    wi, wj, ws = want_low
    keep = ws >= t
    sel = np.isin(gi, rows) | np.isin(gj, rows)
    _check_pairs((gi[sel], gj[sel], gs[sel]), (wi[keep], wj[keep], ws[keep]))
    k = np.arange(0, len(gi), max(1, len(gi) // 4000))
    if len(k):
        s64 = oracle.pair_sims(x, gi[k], gj[k])
        assert np.max(np.abs(gs[k] - s64)) <= SIM_TOL and np.all(s64 >= t)
    return int(sel.sum())


@pytest.fixture(scope="module")
def mixed_1m_40k():
    x = synth.generate("mixed_1m", n=40_000)
    rows = np.arange(0, x.n, 131, dtype=np.int32)
    return x, rows, oracle.rows(x, 0.5, rows)


@pytest.mark.parametrize("precision,p", [(cuapss.PREC_MIXED, 0), (cuapss.PREC_MIXED, 4096),
                                         (cuapss.PREC_FP32, 0)],
                         ids=["mixed-default", "mixed-4096", "fp32-default"])
def test_mixed_1m_shape(mixed_1m_40k, precision, p):
    x, rows, want = mixed_1m_40k
    assert x.d == 1_000_000
    with cuapss.Context(precision=precision, head_width=p) as c:
        for t in (0.5, 0.7, 0.8):
            got = c.run(x, t, capacity=1 << 22)
            if p:
                assert c.last_stats["head_width"] == p
            assert _sampled_check(x, got, t, rows, want) > 0


def test_serve_index_shape_per_row_thresholds():
    cfg = synth.CONFIGS["serve_5m"]
    assert cfg.d == 1 << 20
    x = synth.generate(cfg, n=50_000)
    q = synth.generate(cfg, n=300, row_offset=50_000_000)
    # near-duplicates of index rows among the queries, so that there are pairs
    q = synth.Csr(*_stack(q, x.take(np.arange(0, 50_000, 997))), x.d)
    rng = np.random.default_rng(5)
    t = rng.uniform(0.6, 0.95, size=q.n).astype(np.float32)
    i, j, s = oracle.join(q, x, float(t.min()))
    keep = s >= t[i].astype(np.float64)
    want = (i[keep], j[keep], s[keep])
    assert len(want[0]) > 0
    for precision in (cuapss.PREC_MIXED, cuapss.PREC_FP32):
        with cuapss.Context(precision=precision) as c, cuapss.Index(c, x) as idx:
            _check_pairs(idx.query(q, t), want)


def _stack(a, b):
    rp = np.concatenate([a.rowptr, b.rowptr[1:] + a.rowptr[-1]])
    return rp, np.concatenate([a.col, b.col]), np.concatenate([a.val, b.val])


@pytest.mark.parametrize("precision", [cuapss.PREC_MIXED, cuapss.PREC_FP32], ids=["mixed", "fp32"])
def test_plain_800k_shape_threshold_sweep(precision):
    x = synth.generate("plain_800k", n=60_000)
    rows = np.arange(0, x.n, 149, dtype=np.int32)
    want = oracle.rows(x, 0.5, rows)
    with cuapss.Context(precision=precision) as c:
        for t in (0.5, 0.9):
            assert _sampled_check(x, c.run(x, t, capacity=1 << 22), t, rows, want) > 0


def _all_features_matrix(d, n, rng, dup_every=7):
    """n rows over d features in which every feature occurs at least once;
    every dup_every-th row is a perturbed copy of its predecessor."""
    own_rows = [r for r in range(n) if r % dup_every != dup_every - 1]
    shares = np.array_split(rng.permutation(d), len(own_rows))
    rows, k = [], 0
    for r in range(n):
        if r % dup_every == dup_every - 1:
            f, v = rows[-1]
            rows.append((f, v * rng.uniform(0.95, 1.05, size=len(v))))
            continue
        f = np.unique(np.concatenate([shares[k], rng.integers(0, 2000, size=40)]))
        k += 1
        rows.append((f.astype(np.int32), rng.uniform(0.2, 1.0, size=len(f))))
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(f) for f, _ in rows])
    col = np.concatenate([f for f, _ in rows]).astype(np.int32)
    val = np.concatenate([v / np.linalg.norm(v) for _, v in rows]).astype(np.float32)
    return synth.Csr(rp, col, val, d)


@pytest.mark.parametrize("precision", [cuapss.PREC_MIXED, cuapss.PREC_FP32], ids=["mixed", "fp32"])
def test_tail_feature_keys_at_the_edge(precision):
    p = 64
    d = p + (1 << 20) - 2  # the largest d - p the 20-bit tail keys take
    x = _all_features_matrix(d, 6000, np.random.default_rng(3))
    assert np.unique(x.col).size == d
    want = oracle.apss(x, 0.8)
    assert len(want[0]) > 0
    with cuapss.Context(precision=precision, head_width=p) as c:
        _check_pairs(c.run(x, 0.8, capacity=1 << 20), want)
        assert c.last_stats["head_width"] == p
    # one feature more: rejected, not truncated
    y = synth.Csr(x.rowptr, x.col, x.val, d + 1)
    with cuapss.Context(precision=precision, head_width=p) as c:
        with pytest.raises(cuapss.CuapssError) as e:
            c.run(y, 0.8)
        assert e.value.status == cuapss.EINVAL


@pytest.mark.parametrize("precision", [cuapss.PREC_MIXED, cuapss.PREC_FP32], ids=["mixed", "fp32"])
@pytest.mark.parametrize("tail", [110, 150], ids=["shared-sort", "global-sort"])
def test_chunked_tail_staging_beside_small_blocks(precision, tail):
    # rows 0..127 carry `tail` rare features each: 14,080 or 19,200 tail
    # postings in block 0, more than either tile kernel stages at once
    # (chunked staging), below / above the per-block shared-memory sort's
    # 16,384; every fourth row is followed by three near-duplicates. The
    # other blocks are ordinary rows of the d = 1M workload.
    rng = np.random.default_rng(9 + tail)
    base = synth.generate("mixed_1m", n=3000)
    d = base.d
    heavy, vals = [], []
    for r in range(128):
        if r % 4 == 0:
            f = np.unique(rng.integers(200_000, 240_000, size=tail + 8))[:tail]
            heavy.append(f.astype(np.int32))
            vals.append(rng.uniform(0.2, 1.0, size=len(f)))
        else:
            heavy.append(heavy[-1])
            vals.append(vals[-1] * rng.uniform(0.97, 1.03, size=len(heavy[-1])))
    rp = np.zeros(129, np.int64)
    rp[1:] = np.cumsum([len(f) for f in heavy])
    col = np.concatenate(heavy)
    val = np.concatenate([v / np.linalg.norm(v) for v in vals]).astype(np.float32)
    assert rp[-1] > 12_800
    hrp, hcol, hval = _stack(synth.Csr(rp, col, val, d), base)
    x = synth.Csr(hrp, hcol, hval, d)
    want = oracle.apss(x, 0.7)
    assert len(want[0]) > 0
    with cuapss.Context(precision=precision) as c:
        _check_pairs(c.run(x, 0.7, capacity=1 << 20), want)
