"""Batched self-joins (cuapss_batch_run) against the FP64 oracle run per
instance: the pair set of every instance equals the oracle's at that
instance's threshold, similarities within 1e-6, no pair crosses instances."""
import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6


def oracle_batch(x, inst_ptr, t):
    ii, jj, ss = [], [], []
    for q in range(len(t)):
        a, b = int(inst_ptr[q]), int(inst_ptr[q + 1])
        if b - a < 2:
            continue
        i, j, s = oracle.apss(x.rows(a, b), float(t[q]))
        ii.append(i.astype(np.int64) + a)
        jj.append(j.astype(np.int64) + a)
        ss.append(s)
    if not ii:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
    return np.concatenate(ii), np.concatenate(jj), np.concatenate(ss)


def check(got, want):
    gi, gj, gs = got
    wi, wj, ws = want
    assert len(gi) == len(wi), (len(gi), len(wi))
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gj, wj)
    assert np.max(np.abs(gs.astype(np.float64) - ws), initial=0.0) <= SIM_TOL


def small_batch(seed, k=40, n_lo=2, n_hi=700):
    return synth.generate_batch(k=k, n_lo=n_lo, n_hi=n_hi, t_lo=0.5, t_hi=0.95, seed=seed)


@pytest.fixture(scope="module", params=[cuapss.PREC_MIXED, cuapss.PREC_FP32],
                ids=["mixed", "fp32"])
def ctx(request):
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    with cuapss.Context(precision=request.param) as c:
        yield c


def test_batch_matches_oracle_per_instance(ctx):
    x, ip, t = small_batch(seed=1)
    got = ctx.batch_run(x, ip, t)
    check(got, oracle_batch(x, ip, t))
    # instance of each pair: i and j in the same row range
    qi = np.searchsorted(ip, got[0], side="right")
    qj = np.searchsorted(ip, got[1], side="right")
    np.testing.assert_array_equal(qi, qj)
    assert got[0].size > 0


def test_batch_twice_identical_and_matches_single_runs(ctx):
    x, ip, t = small_batch(seed=2, k=24, n_lo=64, n_hi=3000)
    a = ctx.batch_run(x, ip, t)
    b = ctx.batch_run(x, ip, t)  # same topology: the captured graph is updated
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)
    # the same instances as separate cuapss_run calls
    ii, jj = [], []
    for q in range(len(t)):
        lo, hi = int(ip[q]), int(ip[q + 1])
        i, j, _ = ctx.run(x.rows(lo, hi), float(t[q]))
        ii.append(i.astype(np.int64) + lo)
        jj.append(j.astype(np.int64) + lo)
    np.testing.assert_array_equal(a[0], np.concatenate(ii))
    np.testing.assert_array_equal(a[1], np.concatenate(jj))


def test_batch_all_buckets(ctx):
    # instances in all three size buckets (<= 1024, <= 8192, larger)
    cfg = synth.CONFIGS["batch_instance"]
    parts, ns, ts = [], [300, 9000, 1500, 64, 2000], [0.8, 0.85, 0.7, 0.6, 0.9]
    for q, n in enumerate(ns):
        parts.append(synth.generate(cfg.replace(n=n, stream=100 + q)))
    rp = [np.zeros(1, np.int64)]
    off = 0
    for p in parts:
        rp.append(p.rowptr[1:] + off)
        off += p.nnz
    x = synth.Csr(np.concatenate(rp), np.concatenate([p.col for p in parts]),
                  np.concatenate([p.val for p in parts]), cfg.d)
    ip = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    t = np.array(ts, np.float32)
    got = ctx.batch_run(x, ip, t)
    assert all(ctx.last_bucket_p > 0)
    # the 9000-row instance: compare with the single-join path (oracle-tested)
    want_i, want_j, want_s = [], [], []
    for q in range(len(ns)):
        lo, hi = int(ip[q]), int(ip[q + 1])
        if hi - lo <= 2000:
            i, j, s = oracle.apss(x.rows(lo, hi), float(t[q]))
        else:
            i, j, s = ctx.run(x.rows(lo, hi), float(t[q]))
        want_i.append(i.astype(np.int64) + lo)
        want_j.append(j.astype(np.int64) + lo)
        want_s.append(s.astype(np.float64))
    check(got, (np.concatenate(want_i), np.concatenate(want_j), np.concatenate(want_s)))


def test_batch_edge_instances(ctx):
    # empty and single-row instances, a 129-row instance (two blocks), a
    # 128-row instance (one full block), thresholds at the ends of the range
    cfg = synth.CONFIGS["batch_instance"]
    ns = [0, 1, 129, 0, 128, 2, 1]
    parts = [synth.generate(cfg.replace(n=max(n, 1), stream=7 + q, dup_frac=0.3))
             for q, n in enumerate(ns)]
    parts = [p.rows(0, n) for p, n in zip(parts, ns)]
    rp = [np.zeros(1, np.int64)]
    off = 0
    for p in parts:
        rp.append(p.rowptr[1:] + off)
        off += p.nnz
    x = synth.Csr(np.concatenate(rp), np.concatenate([p.col for p in parts]),
                  np.concatenate([p.val for p in parts]), cfg.d)
    ip = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    t = np.array([0.5, 0.5, 0.3, 0.9, 0.99, 0.1, 0.5], np.float32)
    check(ctx.batch_run(x, ip, t), oracle_batch(x, ip, t))


def test_batch_device_io(ctx):
    import torch
    x, ip, t = small_batch(seed=3, k=16)
    want = ctx.batch_run(x, ip, t)
    dx = {"rowptr": torch.from_numpy(x.rowptr).cuda(), "col": torch.from_numpy(x.col).cuda(),
          "val": torch.from_numpy(x.val).cuda(), "d": x.d}
    cap = len(want[0]) + 1
    out = {"i": torch.empty(cap, dtype=torch.int32, device="cuda"),
           "j": torch.empty(cap, dtype=torch.int32, device="cuda"),
           "sim": torch.empty(cap, dtype=torch.float32, device="cuda")}
    m = ctx.batch_run_device(dx, ip, t, out)
    assert m == len(want[0])
    np.testing.assert_array_equal(out["i"][:m].cpu().numpy(), want[0])
    np.testing.assert_array_equal(out["j"][:m].cpu().numpy(), want[1])
    np.testing.assert_array_equal(out["sim"][:m].cpu().numpy(), want[2])


def test_batch_rejects_bad_arguments(ctx):
    x, ip, t = small_batch(seed=4, k=4)
    bad = ip.copy()
    bad[2] = bad[1] - 1  # decreasing
    with pytest.raises(cuapss.CuapssError) as e:
        ctx.batch_run(x, bad, t)
    assert e.value.status == cuapss.EINVAL
    bad = ip.copy()
    bad[-1] -= 1  # does not cover x
    with pytest.raises(cuapss.CuapssError):
        ctx.batch_run(x, bad, t)
    tb = t.copy()
    tb[1] = 0.0
    with pytest.raises(cuapss.CuapssError):
        ctx.batch_run(x, ip, tb)


def test_batch_fixed_head_width():
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    x, ip, t = small_batch(seed=5, k=12, n_lo=64, n_hi=2500)
    with cuapss.Context(precision=cuapss.PREC_MIXED, head_width=256) as c:
        got = c.batch_run(x, ip, t)
        bp = c.last_bucket_p
    assert set(int(v) for v in bp if v) == {256}
    check(got, oracle_batch(x, ip, t))
