"""Request server (cuapss_server_*): every request's result in the mix of
concurrent batches and appends equals the same query run alone against the
rows it was matched against, within the similarity tolerance -- also when
requests larger than the batch cap run as slices on several lanes."""
import numpy as np
import pytest

import cuapss
from cuapss import synth

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    with cuapss.Context(precision=cuapss.PREC_MIXED) as c:
        yield c


def same(a, b):
    ai, aj, as_ = a
    bi, bj, bs = b
    np.testing.assert_array_equal(ai, bi)
    np.testing.assert_array_equal(aj, bj)
    assert np.max(np.abs(as_.astype(np.float64) - bs.astype(np.float64)), initial=0.0) <= SIM_TOL


def workload(seed, n_requests=60, n_appends=4):
    cfg = synth.CONFIGS["plain_20k"].replace(seed=seed, dup_frac=0.15)
    base = synth.generate(cfg, n=8000)
    rng = np.random.default_rng(seed)
    reqs = []
    off = 8000
    qoff = 500_000
    for k in range(n_requests + n_appends):
        if k % (n_requests // n_appends + 1) == n_requests // n_appends:
            m = int(rng.integers(100, 1500))
            reqs.append(("append", synth.generate(cfg, n=m, row_offset=off), None))
            off += m
        else:
            m = int(np.exp(rng.uniform(0, np.log(300))))
            q = synth.generate(cfg, n=m, row_offset=qoff)
            qoff += m
            t = rng.uniform(0.5, 0.95, size=m).astype(np.float32)
            reqs.append(("query", q, t))
    return base, reqs


@pytest.mark.parametrize("lanes,max_rows,budget", [(3, 512, 16 << 30), (2, 4096, 1),
                                                   (3, 48, 16 << 30)],
                         ids=["three_lanes", "tiny_budget", "sliced"])
def test_mix_equals_alone(ctx, lanes, max_rows, budget):
    base, reqs = workload(seed=lanes)
    with cuapss.Index(ctx, base) as idx:
        results = []
        with cuapss.Server(idx, lanes=lanes, max_batch_rows=max_rows, hbm_budget=budget) as srv:
            tickets = []
            for kind, x, t in reqs:
                tickets.append(srv.submit_append(x) if kind == "append" else srv.submit_query(x, t))
            for tk in tickets:
                results.append(srv.wait(tk, timeout_ms=120_000))
        n_final = idx.info()["rows"]
        assert n_final == base.n + sum(x.n for k, x, _ in reqs if k == "append")
        multi = 0
        for (kind, x, t), (pairs, info) in zip(reqs, results):
            assert info["status"] == cuapss.OK
            if kind == "append":
                continue
            # a request of more than max_rows rows runs as slices of max_rows
            assert info["batch_rows"] >= min(x.n, max_rows)
            multi += info["batch_rows"] > min(x.n, max_rows)
            # alone: the same query against the index now, restricted to the
            # rows this request was matched against
            ai, aj, as_ = idx.query(x, t)
            keep = aj < info["index_rows"]
            same(pairs, (ai[keep], aj[keep], as_[keep]))
            assert info["latency_ms"] >= info["queue_ms"] >= 0.0
        if budget > 1 and max_rows < 4096:
            assert multi > 0  # requests shared batches


def test_server_rejects_bad_requests(ctx):
    base, reqs = workload(seed=11, n_requests=5, n_appends=1)
    with cuapss.Index(ctx, base) as idx, cuapss.Server(idx, lanes=1) as srv:
        q = reqs[0][1]
        with pytest.raises(cuapss.CuapssError):
            srv.submit_query(q, np.zeros(q.n, np.float32))
        bad = synth.Csr(q.rowptr, q.col, q.val, q.d + 5)
        tk = srv.submit_query(bad, np.full(q.n, 0.7, np.float32))
        with pytest.raises(cuapss.CuapssError) as e:
            srv.wait(tk)
        assert e.value.status == cuapss.EINVAL
        # the server keeps serving
        tk = srv.submit_query(q, np.full(q.n, 0.7, np.float32))
        pairs, info = srv.wait(tk)
        assert info["status"] == cuapss.OK
