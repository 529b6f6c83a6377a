"""GPU parity of the explicit rare-feature pairs of self-joins, through the C
ABI, against the FP64 oracle.

Features that occur in at most C rows have their pairs enumerated and added
to the tiles' tail accumulators instead of being probed. The threshold is
normally chosen with the head width by the cost model; these tests force it
(the rare_max_count option) so that every threshold's records are checked:

* the n = d = 1M workload's distribution at 8,000 rows, C in {16, 256, 2048}
  and none, both precisions: the same pair set as the oracle and as the run
  without explicit pairs;
* 256 rows whose 2,000 shared rare features give one tile about 1,000
  records, more than the mixed kernel holds in registers (the rest are read
  where they are added);
* the cost model's own choice at 40,000 rows takes explicit pairs (below
  32,768 rows it plans none);
* 1.1M rows, whose tile rows span more J blocks than one counting CTA
  covers;
* row-block shards, each building the pairs of its own tile rows."""
import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6
PRECISIONS = [(cuapss.PREC_MIXED, "mixed"), (cuapss.PREC_FP32, "fp32")]


def _check(got, want):
    gi, gj, gs = got
    wi, wj, ws = want
    assert len(gi) == len(wi), f"pair count {len(gi)} != oracle {len(wi)}"
    assert np.array_equal(gi, wi) and np.array_equal(gj, wj)
    if len(gs):
        err = float(np.max(np.abs(gs.astype(np.float64) - ws)))
        assert err <= SIM_TOL, f"max |sim - fp64| = {err}"


@pytest.fixture(scope="module")
def zipf8k():
    x = synth.generate("mixed_1m", n=8000)
    return x, oracle.apss(x, 0.5)


@pytest.mark.parametrize("precision,name", PRECISIONS, ids=[n for _, n in PRECISIONS])
@pytest.mark.parametrize("rare", [-1, 16, 256, 2048])
def test_forced_thresholds_match_oracle(zipf8k, precision, name, rare):
    x, want = zipf8k
    with cuapss.Context(precision=precision, rare_max_count=rare) as c:
        got = c.run(x, 0.5, capacity=1 << 20)
        st = c.last_stats
    _check(got, want)
    if rare < 0:
        assert st["explicit_pairs"] == 0 and st["rare_max_count"] == 0
    else:
        counts = np.bincount(x.col, minlength=x.d)
        rare_f = counts[(counts >= 2) & (counts <= rare)]
        assert st["rare_max_count"] == rare
        # every pair of each rare feature (minus those the head keeps)
        assert 0 < st["explicit_pairs"] <= int((rare_f * (rare_f - 1) // 2).sum())


def _shared_rare_rows(rng, n=256, shared=2000, common=100):
    feats = [[] for _ in range(n)]
    for f in range(shared):  # rare features 1000 .. : two rows each
        a, b = rng.choice(n, size=2, replace=False)
        feats[a].append(1000 + f)
        feats[b].append(1000 + f)
    for r in range(n):  # a few common features (ids < common)
        feats[r].extend(rng.choice(common, size=12, replace=False).tolist())
    rp = np.zeros(n + 1, np.int64)
    cols, vals = [], []
    for r in range(n):
        f = np.unique(np.asarray(feats[r], np.int32))
        v = rng.uniform(0.1, 1.0, size=len(f))
        cols.append(f)
        vals.append(v / np.linalg.norm(v))
        rp[r + 1] = rp[r] + len(f)
    return synth.Csr(rp, np.concatenate(cols), np.concatenate(vals).astype(np.float32),
                     1000 + shared)


@pytest.mark.parametrize("precision,name", PRECISIONS, ids=[n for _, n in PRECISIONS])
def test_tile_with_many_records(precision, name):
    x = _shared_rare_rows(np.random.default_rng(21))
    want = oracle.apss(x, 0.2)
    assert len(want[0]) > 0
    with cuapss.Context(precision=precision, head_width=64, rare_max_count=16) as c:
        got = c.run(x, 0.2, capacity=1 << 18)
        st = c.last_stats
    _check(got, want)
    assert st["explicit_pairs"] == 2000  # one pair per shared feature; 3 tiles


def test_model_takes_explicit_pairs():
    x = synth.generate("mixed_1m", n=40000)
    rows = np.random.default_rng(5).choice(x.n, size=200, replace=False)
    wi, wj, ws = oracle.rows(x, 0.7, rows)
    with cuapss.Context(precision=cuapss.PREC_MIXED) as c:
        gi, gj, gs = c.run(x, 0.7, capacity=1 << 20)
        st = c.last_stats
    assert st["explicit_pairs"] > 0 and st["rare_max_count"] >= 16
    # the host planner makes the same choice from the posting counts
    plan = cuapss.plan_self_join(x)
    assert plan["head_width"] == st["head_width"]
    assert plan["rare_max_count"] == st["rare_max_count"]
    assert 0 < st["explicit_pairs"] <= plan["explicit_pairs"]
    with cuapss.Context(precision=cuapss.PREC_MIXED) as c:
        c.run(x.rows(0, 20000), 0.7)
        assert c.last_stats["explicit_pairs"] == 0  # too small to plan
    sel = np.isin(gi, rows) | np.isin(gj, rows)
    _check((gi[sel], gj[sel], gs[sel]), (wi, wj, ws))


def test_tile_rows_past_one_counting_range():
    # 1.1M rows: 8,594 row blocks, more than the 8,192 J blocks one counting
    # / placement CTA covers, so the tile rows are split over two CTAs (the
    # second starts above the diagonal and finds each posting's first pair
    # in its range by binary search)
    x = synth.generate("mixed_1m", n=1_100_000)
    rows = np.random.default_rng(8).choice(x.n, size=64, replace=False)
    rows = np.concatenate([rows, [x.n - 1, 0, 8192 * 128 + 5]]).astype(np.int32)
    wi, wj, ws = oracle.rows(x, 0.5, rows)
    assert len(wi) > 500
    with cuapss.Context(precision=cuapss.PREC_MIXED, head_width=1024, rare_max_count=128) as c:
        gi, gj, gs = c.run(x, 0.5, capacity=1 << 25)
        st = c.last_stats
    assert st["rare_max_count"] == 128 and st["explicit_pairs"] > 0
    sel = np.isin(gi, rows) | np.isin(gj, rows)
    _check((gi[sel], gj[sel], gs[sel]), (wi, wj, ws))


@pytest.mark.parametrize("precision,name", PRECISIONS, ids=[n for _, n in PRECISIONS])
def test_shards_with_explicit_pairs(zipf8k, precision, name):
    # each row-block shard builds the explicit pairs of its own tile rows;
    # the shards' union equals the whole join and the oracle, bit for bit
    x, want = zipf8k
    with cuapss.Context(precision=precision, rare_max_count=256) as c:
        full = c.run(x, 0.5, capacity=1 << 20)
        whole = c.last_stats["explicit_pairs"]
        _check(full, want)
        for nshards in (2, 3):
            parts, kept = [], 0
            for s in range(nshards):
                parts.append(c.run_shard(x, 0.5, s, nshards, capacity=1 << 20))
                assert c.last_stats["rare_max_count"] == 256
                kept += c.last_stats["explicit_pairs"]
                assert np.all((parts[-1][0] // 128) % nshards == s)
            assert kept == whole  # every pair in exactly one shard
            key = np.concatenate([p[0].astype(np.int64) * x.n + p[1] for p in parts])
            order = np.argsort(key)
            assert np.array_equal(key[order], full[0].astype(np.int64) * x.n + full[1])
            assert np.array_equal(np.concatenate([p[2] for p in parts])[order], full[2])
