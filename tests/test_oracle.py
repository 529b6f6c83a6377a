"""CPU oracle checks: pinned against the reference's own CPU search (golden
fixture), hand-built known answers, and a dense brute force."""
import json
import os

import numpy as np
import pytest

from cuapss import synth
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_cpu_search.json")


def _dense(x):
    m = np.zeros((x.n, x.d), np.float64)
    for i in range(x.n):
        a, b = x.rowptr[i], x.rowptr[i + 1]
        m[i, x.col[a:b]] = x.val[a:b]
    return m


def _csr_from_rows(rows, d):
    rp = [0]
    col, val = [], []
    for r in rows:
        for c, v in sorted(r):
            col.append(c)
            val.append(v)
        rp.append(len(col))
    return synth.Csr(np.array(rp), np.array(col, np.int32), np.array(val, np.float32), d)


@pytest.mark.parametrize("case", json.load(open(GOLDEN))["cases"], ids=lambda c: c["name"])
def test_oracle_matches_reference_cpu_search(case):
    """The reference's InvertedIndex_search (main.cu:104-141), compiled from
    its own source, counted these pairs at its hard-coded t = 0.8."""
    from tests.golden.make_golden import digest
    x = synth.generate(case["config"], **case["overrides"])
    assert digest(x) == case["input_sha256"], "generator output changed"
    b = x.rows(*case["b_rows"])
    e = x.rows(*case["e_rows"])
    i, j, s = oracle.join(b, e, case["t"])
    assert len(i) == case["ref_sum_pair"]
    assert case["closest_sim_to_t"] > 1e-5  # the FP32 reference cannot flip a pair


def test_known_answers():
    v = np.float32(0.6)
    w = np.float32(0.8)
    rows = [
        [(1, v), (5, w)],          # 0
        [(1, v), (5, w)],          # 1 identical to 0 -> 1.0
        [(2, np.float32(1.0))],    # 2 disjoint from 0 -> 0
        [(1, w), (5, v)],          # 3 with 0: 0.6*0.8*2 = 0.96
        [(5, np.float32(1.0))],    # 4 with 0: 0.8 exactly representable product
    ]
    x = _csr_from_rows(rows, 8)
    i, j, s = oracle.apss(x, 0.5)
    got = {(int(a), int(b)): float(c) for a, b, c in zip(i, j, s)}
    assert got[(0, 1)] == pytest.approx(float(v) * float(v) + float(w) * float(w), abs=0)
    assert (0, 2) not in got
    assert got[(0, 3)] == float(v) * float(w) + float(w) * float(v)
    t_exact = float(w)  # pair (0,4) has similarity exactly float(w)
    i, j, s = oracle.apss(x, t_exact)
    assert (0, 4) in set(zip(i.tolist(), j.tolist()))
    i, j, s = oracle.apss(x, np.nextafter(t_exact, 2.0))
    assert (0, 4) not in set(zip(i.tolist(), j.tolist()))


def test_oracle_vs_dense_bruteforce():
    x = synth.generate("plain_20k", n=600)
    m = _dense(x)
    g = m @ m.T
    for t in (0.3, 0.6, 0.9):
        iu = np.triu_indices(x.n, 1)
        sel = g[iu] >= t
        want = set(zip(iu[0][sel].tolist(), iu[1][sel].tolist()))
        i, j, s = oracle.apss(x, t)
        assert set(zip(i.tolist(), j.tolist())) == want
        assert np.max(np.abs(s - g[i, j])) < 1e-12
        assert np.all(np.diff(i.astype(np.int64) * x.n + j) > 0)  # sorted, unique


def test_rows_oracle_consistent_with_apss():
    x = synth.generate("plain_20k", n=3000)
    i, j, s = oracle.apss(x, 0.7)
    rows = np.arange(0, 3000, 7)
    ri, rj, rs = oracle.rows(x, 0.7, rows)
    sel = np.isin(i, rows) | np.isin(j, rows)
    assert np.array_equal(ri, i[sel]) and np.array_equal(rj, j[sel])
    assert np.array_equal(rs, s[sel])  # bit-identical sums (same order)


def test_index_ref_and_remap():
    x = synth.generate("plain_20k", n=2000)
    p = 4096
    dim_ptr, rows, vals = oracle.index_ref(x, p)
    m = _dense(x)
    for f in (p, p + 1, 5000, 9999):
        nz = np.nonzero(m[:, f])[0]
        assert np.array_equal(rows[dim_ptr[f]:dim_ptr[f + 1]], nz)
        assert np.array_equal(vals[dim_ptr[f]:dim_ptr[f + 1]], m[nz, f].astype(np.float32))
    assert dim_ptr[p] == 0 and dim_ptr[-1] == int((x.col >= p).sum())
    perm, counts = oracle.feature_remap(x)
    want_counts = np.bincount(x.col, minlength=x.d)
    assert np.array_equal(counts, want_counts)
    order = np.lexsort((np.arange(x.d), -want_counts))
    assert np.array_equal(perm[order], np.arange(x.d))


def test_cpu_hybrid_counts_match_oracle():
    x = synth.generate("plain_20k", n=4000)
    for t in (0.5, 0.9):
        want = len(oracle.apss(x, t)[0])
        got, _, _ = oracle.cpu_hybrid(x, t, 64, 0, x.n)
        assert abs(got - want) <= max(2, want // 1000)


def test_batch_generator_layout():
    x, ip, t = synth.generate_batch(k=50, n_lo=64, n_hi=2000, seed=9)
    assert ip[0] == 0 and ip[-1] == x.n and np.all(np.diff(ip) >= 64)
    assert np.all(np.diff(ip) <= 2000) and t.shape == (50,)
    assert np.all((t >= 0.6) & (t <= 0.95))
    nrm = np.sqrt(np.add.reduceat(x.val.astype(np.float64) ** 2, x.rowptr[:-1]))
    assert np.allclose(nrm, 1.0, atol=1e-5)
    # instance rows come from independent streams over one vocabulary: the
    # same seed gives the same batch, stream 0 is the plain stream
    x2, ip2, t2 = synth.generate_batch(k=50, n_lo=64, n_hi=2000, seed=9)
    np.testing.assert_array_equal(x.col, x2.col)
    a = synth.generate("batch_instance", n=100)
    b = synth.generate("batch_instance", n=100, stream=0)
    np.testing.assert_array_equal(a.col, b.col)
    c = synth.generate("batch_instance", n=100, stream=3)
    assert not np.array_equal(a.col[:50], c.col[:50])
