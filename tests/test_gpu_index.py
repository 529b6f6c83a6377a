"""Resident index (cuapss_index_*): query batches with per-query thresholds
against the FP64 oracle cross-join, appends and segment merges, concurrency
of queries from two contexts."""
import threading

import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6


def oracle_query(q, x, t):
    """Pairs (query row, index row) with FP64 sim >= t[i]."""
    i, j, s = oracle.join(q, x, float(np.min(t)))
    keep = s >= t[i].astype(np.float64)
    return i[keep].astype(np.int64), j[keep].astype(np.int64), s[keep]


def check(got, want):
    gi, gj, gs = got
    wi, wj, ws = want
    assert len(gi) == len(wi), (len(gi), len(wi))
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gj, wj)
    assert np.max(np.abs(gs.astype(np.float64) - ws), initial=0.0) <= SIM_TOL


def data(n_index=6000, n_q=300, seed=0):
    cfg = synth.CONFIGS["plain_20k"].replace(seed=seed, dup_frac=0.1)
    x = synth.generate(cfg, n=n_index)
    # queries: fresh rows of the same stream (near-duplicates of index rows)
    q = synth.generate(cfg, n=n_q, row_offset=n_index)
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.5, 0.9, size=q.n).astype(np.float32)
    return x, q, t


@pytest.fixture(scope="module", params=[cuapss.PREC_MIXED, cuapss.PREC_FP32],
                ids=["mixed", "fp32"])
def ctx(request):
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    with cuapss.Context(precision=request.param) as c:
        yield c


def test_query_matches_oracle(ctx):
    x, q, t = data()
    with cuapss.Index(ctx, x) as idx:
        got = idx.query(q, t)
        assert got[0].size > 0
        check(got, oracle_query(q, x, t))
        info = idx.info()
        assert info["rows"] == x.n and info["segments"] == 1


def test_query_edge_sizes(ctx):
    x, q, t = data(n_index=1000, n_q=130, seed=3)
    with cuapss.Index(ctx, x) as idx:
        for n in (0, 1, 127, 128, 129):
            qq = q.rows(0, n)
            got = idx.query(qq, t[:n]) if n else idx.query(qq, np.zeros(0, np.float32))
            if n == 0:
                assert got[0].size == 0
            else:
                check(got, oracle_query(qq, x, t[:n]))


def test_appends_and_merges(ctx):
    cfg = synth.CONFIGS["plain_20k"].replace(seed=5, dup_frac=0.1)
    base = synth.generate(cfg, n=3000)
    with cuapss.Index(ctx, base) as idx:
        rows = [base]
        off = 3000
        for k, m in enumerate([200, 129, 1, 700, 1500, 64, 3000]):
            add = synth.generate(cfg, n=m, row_offset=off)
            off += m
            idx.append(add)
            rows.append(add)
            full = synth.Csr(
                np.concatenate([[0]] + [r.rowptr[1:] + sum(z.nnz for z in rows[:i])
                                        for i, r in enumerate(rows)]),
                np.concatenate([r.col for r in rows]), np.concatenate([r.val for r in rows]),
                cfg.d)
            info = idx.info()
            assert info["rows"] == full.n
            assert 1 <= info["segments"] <= 2 + int(np.log2(full.n))
            q = synth.generate(cfg, n=150, row_offset=100_000 + 1000 * k)
            t = np.full(q.n, 0.6, np.float32)
            check(idx.query(q, t), oracle_query(q, full, t))


def test_queries_from_two_contexts(ctx):
    x, q, t = data(n_index=5000, n_q=400, seed=7)
    want = oracle_query(q, x, t)
    with cuapss.Index(ctx, x) as idx, cuapss.Context() as c2:
        results = {}

        def run(name, c):
            results[name] = [idx.query(q, t, ctx=c) for _ in range(3)]

        th = [threading.Thread(target=run, args=("a", ctx)),
              threading.Thread(target=run, args=("b", c2))]
        for h in th:
            h.start()
        for h in th:
            h.join()
        for name in ("a", "b"):
            for got in results[name]:
                check(got, want)


def test_query_rejects_bad_arguments(ctx):
    x, q, t = data(n_index=500, n_q=10, seed=9)
    with cuapss.Index(ctx, x) as idx:
        with pytest.raises(cuapss.CuapssError):
            idx.query(q, np.zeros(q.n, np.float32))
        bad = synth.Csr(q.rowptr, q.col, q.val, q.d + 1)
        with pytest.raises(cuapss.CuapssError):
            idx.query(bad, t)
