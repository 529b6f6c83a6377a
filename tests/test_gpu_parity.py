"""GPU parity: the CUDA path, called through the C ABI, against the FP64
oracle. Pair sets must be equal; reported similarities within 1e-6 of the
oracle's FP64 value (tolerance stated by the exactness contract)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

SIM_TOL = 1e-6  # |reported - FP64| bound of the exactness contract


def _check_pairs(got, want, tol=SIM_TOL):
    gi, gj, gs = got
    wi, wj, ws = want
    assert len(gi) == len(wi), f"pair count {len(gi)} != oracle {len(wi)}"
    assert np.array_equal(gi, wi) and np.array_equal(gj, wj)
    if len(gs):
        err = np.max(np.abs(gs.astype(np.float64) - ws))
        assert err <= tol, f"max |sim - fp64| = {err}"


@pytest.mark.parametrize("t", [0.9, 0.7, 0.5])
def test_plain_20k_matches_oracle(gpu_ctx, t):
    x = synth.generate("plain_20k")
    got = gpu_ctx.run(x, t)
    _check_pairs(got, oracle.apss(x, t))
    st = gpu_ctx.last_stats
    assert st["pairs"] == len(got[0]) and st["candidates"] >= st["pairs"]


@pytest.mark.parametrize("p", [32, 64, 128, 256])
def test_head_widths(p):
    x = synth.generate("batch_instance", n=3000, seed=3)
    with cuapss.Context(head_width=p) as c:
        got = c.run(x, 0.6)
        assert c.last_stats["head_width"] == p
    _check_pairs(got, oracle.apss(x, 0.6))


def test_no_remap_and_reference_head_rule():
    x = synth.generate("plain_20k", n=5000)
    with cuapss.Context(remap=False, head_width=4096) as c:
        got = c.run(x, 0.8)
    _check_pairs(got, oracle.apss(x, 0.8))


def test_known_answers(gpu_ctx):
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
        _check_pairs(gpu_ctx.run(x, t), oracle.apss(x, t))


def test_edge_sizes(gpu_ctx):
    full = synth.generate("plain_20k", n=700)
    for n in (0, 1, 2, 127, 128, 129, 255, 257, 700):
        x = full.rows(0, n)
        _check_pairs(gpu_ctx.run(x, 0.5), oracle.apss(x, 0.5))


def test_duplicate_heavy_and_single_entry_rows(gpu_ctx):
    # every row identical or a single feature: many exact ties at 1.0
    d = 50
    rows = 300
    rp = np.arange(rows + 1, dtype=np.int64)
    col = (np.arange(rows) % 7).astype(np.int32)
    val = np.ones(rows, np.float32)
    x = synth.Csr(rp, col, val, d)
    _check_pairs(gpu_ctx.run(x, 1.0), oracle.apss(x, 1.0))
    _check_pairs(gpu_ctx.run(x, 0.999), oracle.apss(x, 0.999))


def test_cross_join_matches_oracle(gpu_ctx):
    x = synth.generate("plain_20k", n=9000)
    a, b = x.rows(0, 3000), x.rows(3000, 9000)
    for t in (0.8, 0.5):
        _check_pairs(gpu_ctx.join(a, b, t), oracle.join(a, b, t))


def test_determinism(gpu_ctx):
    x = synth.generate("plain_20k", n=8000)
    r1 = gpu_ctx.run(x, 0.6)
    r2 = gpu_ctx.run(x, 0.6)
    for u, v in zip(r1, r2):
        assert np.array_equal(u, v)


def test_invalid_inputs_rejected(gpu_ctx):
    x = synth.generate("plain_20k", n=200)
    bad = synth.Csr(x.rowptr.copy(), x.col.copy(), x.val.copy(), x.d)
    bad.col[1], bad.col[0] = bad.col[0], bad.col[1]  # unsorted row
    with pytest.raises(cuapss.CuapssError) as e:
        gpu_ctx.run(bad, 0.5)
    assert e.value.status == cuapss.EINVAL
    bad = synth.Csr(x.rowptr.copy(), x.col.copy(), x.val.copy(), x.d)
    bad.col[5] = x.d + 3  # out of range
    with pytest.raises(cuapss.CuapssError) as e:
        gpu_ctx.run(bad, 0.5)
    assert e.value.status == cuapss.EINVAL
    bad = synth.Csr(x.rowptr.copy(), x.col.copy(), x.val * 1.5, x.d)  # not normalised
    with pytest.raises(cuapss.CuapssError) as e:
        gpu_ctx.run(bad, 0.5)
    assert e.value.status == cuapss.EINVAL
    bad = synth.Csr(x.rowptr.copy(), x.col.copy(), x.val.copy(), x.d)
    bad.rowptr[3] = bad.rowptr[5] + 10  # rowptr not monotone
    with pytest.raises(cuapss.CuapssError) as e:
        gpu_ctx.run(bad, 0.5)
    assert e.value.status == cuapss.EINVAL
    with pytest.raises(cuapss.CuapssError) as e:
        gpu_ctx.run(x, 0.0)
    assert e.value.status == cuapss.EINVAL


def test_overflow_reports_required_capacity(gpu_ctx):
    import ctypes
    x = synth.generate("plain_20k", n=6000)
    want = oracle.apss(x, 0.5)
    d, keep = cuapss._desc(x)
    cap = max(1, len(want[0]) // 2)
    oi = np.empty(cap, np.int32)
    oj = np.empty(cap, np.int32)
    os_ = np.empty(cap, np.float32)
    pr = cuapss.PairsDesc(oi.ctypes.data, oj.ctypes.data, os_.ctypes.data, cap, 0, 0)
    s = cuapss.lib().cuapss_run(gpu_ctx._h, ctypes.byref(d), ctypes.c_float(0.5),
                                ctypes.byref(pr), None)
    assert s == cuapss.EOVERFLOW and pr.count == len(want[0])


def test_device_pointers_in_and_out(gpu_ctx):
    import torch
    x = synth.generate("plain_20k", n=5000)
    dev = {"rowptr": torch.from_numpy(x.rowptr).cuda(), "col": torch.from_numpy(x.col).cuda(),
           "val": torch.from_numpy(x.val).cuda(), "d": x.d}
    want = oracle.apss(x, 0.6)
    cap = len(want[0]) + 10
    out = {"i": torch.empty(cap, dtype=torch.int32, device="cuda"),
           "j": torch.empty(cap, dtype=torch.int32, device="cuda"),
           "sim": torch.empty(cap, dtype=torch.float32, device="cuda")}
    m = gpu_ctx.run_device(dev, 0.6, out)
    got = (out["i"][:m].cpu().numpy(), out["j"][:m].cpu().numpy(), out["sim"][:m].cpu().numpy())
    _check_pairs(got, want)


def test_build_index_matches_reference_semantics(gpu_ctx):
    x = synth.generate("plain_20k", n=6000)
    for p in (4096, 0, 9000):
        dp, rows, vals = gpu_ctx.build_index(x, p)
        wdp, wrows, wvals = oracle.index_ref(x, p)
        assert np.array_equal(dp, wdp)
        assert np.array_equal(rows, wrows) and np.array_equal(vals, wvals)


def test_build_index_matches_reference_kernels(gpu_ctx):
    """The reference's own generate_index_ptr4 + construct_Index2, compiled
    from its source into oracle/_ref/ref_index, on the same input."""
    exe = oracle.ref_index_path()
    if exe is None:
        pytest.skip("oracle/_ref/ref_index not built")
    x = synth.generate("plain_20k", n=6000)
    with tempfile.TemporaryDirectory() as td:
        pin, pout = os.path.join(td, "x.csr"), os.path.join(td, "x.idx")
        x.save(pin)
        subprocess.run([exe, pin, pout], check=True, capture_output=True)
        with open(pout, "rb") as f:
            d, total = np.fromfile(f, np.int64, 2)
            max_dim = 198456
            rdp = np.fromfile(f, np.int32, max_dim + 1)
            rrows = np.fromfile(f, np.int32, total)
            rvals = np.fromfile(f, np.float32, total)
    dp, rows, vals = gpu_ctx.build_index(x, 4096)
    assert np.array_equal(dp, rdp[:x.d + 1])
    assert np.all(rdp[x.d:] == rdp[x.d])
    assert np.array_equal(rows, rrows) and np.array_equal(vals, rvals)


def test_feature_remap_matches_oracle(gpu_ctx):
    x = synth.generate("plain_800k", n=20000)
    perm, counts = gpu_ctx.feature_remap(x)
    wperm, wcounts = oracle.feature_remap(x)
    assert np.array_equal(counts, wcounts) and np.array_equal(perm, wperm)


def test_scale_sampled_rows(gpu_ctx):
    """Larger instance: sampled rows checked exactly against the FP64 oracle
    (the full oracle would take too long), plus size-independent checks."""
    x = synth.generate("plain_800k", n=60000)
    t = 0.7
    gi, gj, gs = gpu_ctx.run(x, t, capacity=1 << 20)
    assert np.all(gi < gj)
    key = gi.astype(np.int64) * x.n + gj
    assert np.all(np.diff(key) > 0)
    rows = np.arange(0, x.n, 97, dtype=np.int32)
    wi, wj, ws = oracle.rows(x, t, rows)
    sel = np.isin(gi, rows) | np.isin(gj, rows)
    _check_pairs((gi[sel], gj[sel], gs[sel]), (wi, wj, ws))
    # every reported similarity against FP64 on a sample of all pairs
    k = np.arange(0, len(gi), max(1, len(gi) // 5000))
    s64 = oracle.pair_sims(x, gi[k], gj[k])
    assert np.max(np.abs(gs[k] - s64)) <= SIM_TOL and np.all(s64 >= t)


@pytest.mark.parametrize("precision", [cuapss.PREC_MIXED, cuapss.PREC_FP32], ids=["mixed", "fp32"])
def test_row_lengths_across_sort_paths(precision):
    # rows of 1..32 entries (warp sort), 33..4096 (block sort) and > 4096
    # (the global sort fallback), with near-duplicates of the long rows
    rng = np.random.default_rng(7)
    d = 12_000
    lens = [1, 2, 31, 32, 33, 64, 65, 1000, 4096, 4097, 6000]
    rows = []
    for L in lens:
        f = np.sort(rng.choice(d, size=L, replace=False)).astype(np.int32)
        v = rng.uniform(0.5, 1.5, size=L)
        rows.append((f, v))
        g = f.copy()
        w = v * rng.uniform(0.95, 1.05, size=L)
        rows.append((g, w))  # a near-duplicate of it
    for _ in range(200):
        L = int(rng.integers(1, 80))
        rows.append((np.sort(rng.choice(d, size=L, replace=False)).astype(np.int32),
                     rng.uniform(0.5, 1.5, size=L)))
    rp = np.zeros(len(rows) + 1, np.int64)
    rp[1:] = np.cumsum([len(f) for f, _ in rows])
    col = np.concatenate([f for f, _ in rows])
    val = np.concatenate([(v / np.linalg.norm(v)) for _, v in rows]).astype(np.float32)
    x = synth.Csr(rp, col, val, d)
    with cuapss.Context(precision=precision) as c:
        for t in (0.3, 0.9):
            got = c.run(x, t)
            _check_pairs(got, oracle.apss(x, t))
            assert got[0].size > 0


@pytest.mark.parametrize("extra", [0, 1], ids=["16384", "16385"])
def test_block_tail_at_shared_sort_capacity(extra):
    # Every row holds head features 0..63 (count 256, the whole head at
    # p = 64) and 128 tail features: each 128-row block has exactly 16,384
    # tail postings, the capacity of the per-block shared-memory sort; one
    # extra posting in the second block sends the build to the global radix
    # sort instead. Both must give the oracle's pairs.
    rng = np.random.default_rng(11 + extra)
    d = 64 + 20_000
    rows = []
    for r in range(256):
        nt = 128 + (1 if (extra and r == 200) else 0)
        f = np.concatenate([np.arange(64), 64 + rng.choice(20_000, size=nt, replace=False)])
        rows.append(np.sort(f).astype(np.int32))
    rp = np.zeros(len(rows) + 1, np.int64)
    rp[1:] = np.cumsum([len(f) for f in rows])
    col = np.concatenate(rows)
    val = np.where(col < 64, rng.uniform(1.0, 2.0, size=len(col)),
                   rng.uniform(0.2, 1.0, size=len(col)))
    for r in range(256):
        seg = slice(rp[r], rp[r + 1])
        val[seg] /= np.linalg.norm(val[seg])
    x = synth.Csr(rp, col, val.astype(np.float32), d)
    for precision in (cuapss.PREC_MIXED, cuapss.PREC_FP32):
        with cuapss.Context(precision=precision, head_width=64) as c:
            got = c.run(x, 0.72)
            assert c.last_stats["head_width"] == 64
        _check_pairs(got, oracle.apss(x, 0.72))
        assert got[0].size > 0
