"""The reference-signature shim (include/cuapss_compat.h): tile-ELL layout
conversion (CPU), exported symbols (CPU), and similarity_join_device's pair
counts per partition pair against the FP64 oracle (GPU)."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

import cuapss
from cuapss import synth

# C++ symbol of similarity_join_device with the reference's signature
# (similarity_search.h:3-14): 24 tile-ELL pointers, 8 norm arrays, 24 ints,
# 3 schedule pointers.
MANGLED = ("_Z22similarity_join_devicePiPfS_S_S0_S_S_S0_S_S_S0_S_S_S0_S_S_S0_S_S_S0_S_S_S0_"
           "S_S0_S0_S0_S0_S0_S0_S0_S0_iiiiiiiiiiiiiiiiiiiiiiiiS_S_S_")


def to_tile_ell(x, rng=None):
    """The reference loader's layout: tiles of 32 vectors, entry j of vector v
    at tile_start[v // 32] + v % 32 + 32 j, width = longest vector of the tile,
    unused slots -1 (entries optionally shuffled within each vector)."""
    n = x.n
    ntile = (n + 31) // 32
    lens = np.diff(x.rowptr)
    widths = [int(lens[32 * k:32 * k + 32].max()) if n else 0 for k in range(ntile)]
    ts = np.zeros(ntile + 1, np.int32)
    ts[1:] = np.cumsum(np.array(widths, np.int64) * 32)
    dim = np.full(max(int(ts[-1]), 1), -1, np.int32)
    feat = np.zeros(max(int(ts[-1]), 1), np.float32)
    for v in range(n):
        a, b = int(x.rowptr[v]), int(x.rowptr[v + 1])
        order = np.arange(b - a) if rng is None else rng.permutation(b - a)
        base = ts[v // 32] + v % 32
        for j, e in enumerate(order):
            dim[base + 32 * j] = x.col[a + e]
            feat[base + 32 * j] = x.val[a + e]
    return dim, feat, ts


def convert(dim, feat, ts, n):
    L = cuapss.lib()
    f = L.cuapss_compat_tile_ell_to_csr
    f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3
    f.restype = ctypes.c_int64
    rp = np.zeros(n + 1, np.int64)
    col = np.zeros(max(len(dim), 1), np.int32)
    val = np.zeros(max(len(dim), 1), np.float32)
    m = f(dim.ctypes.data, feat.ctypes.data, ts.ctypes.data, n, len(ts) - 1, rp.ctypes.data,
          col.ctypes.data, val.ctypes.data)
    return m, rp, col[:max(m, 0)], val[:max(m, 0)]


def test_tile_ell_round_trip():
    x = synth.generate("plain_20k", n=517)
    dim, feat, ts = to_tile_ell(x, np.random.default_rng(0))
    m, rp, col, val = convert(dim, feat, ts, x.n)
    assert m == x.nnz
    np.testing.assert_array_equal(rp, x.rowptr)
    np.testing.assert_array_equal(col, x.col)
    np.testing.assert_array_equal(val, x.val)


def test_tile_ell_rejects_malformed():
    x = synth.generate("plain_20k", n=40)
    dim, feat, ts = to_tile_ell(x)
    bad = dim.copy()
    bad[ts[0] + 32] = bad[ts[0]]  # vector 0 repeats its first feature
    assert convert(bad, feat, ts, x.n)[0] == -1
    ts2 = ts.copy()
    ts2[1] += 1  # tile width not a whole number of 32-slot columns
    assert convert(dim, feat, ts2, x.n)[0] == -1


def test_compat_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", cuapss.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert MANGLED in names
    for n in ("cuapss_compat_set_threshold", "cuapss_compat_counts",
              "cuapss_compat_tile_ell_to_csr"):
        assert n in names


@pytest.mark.gpu
def test_similarity_join_device_counts(capfd):
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    from oracle import oracle
    cfg = synth.CONFIGS["plain_20k"].replace(dup_frac=0.2)
    sizes = [300, 257, 0, 32, 1, 500, 100, 64]
    parts, off = [], 0
    for s in sizes:
        parts.append(synth.generate(cfg, n=max(s, 1), row_offset=off).rows(0, s))
        off += s
    t = 0.6
    L = cuapss.lib()
    L.cuapss_compat_set_threshold.argtypes = [ctypes.c_float]
    L.cuapss_compat_set_threshold(t)
    layouts = [to_tile_ell(p) for p in parts]
    args, keep = [], []
    for dim, feat, ts in layouts:
        keep += [dim, feat, ts]
        args += [dim.ctypes.data, feat.ctypes.data, ts.ctypes.data]
    norms = [np.zeros(max(s, 1), np.float32) for s in sizes]
    args += [a.ctypes.data for a in norms]
    for (dim, feat, ts), s in zip(layouts, sizes):
        args += [s, len(dim), len(ts) - 1]
    sched = np.zeros(1, np.int32)
    args += [sched.ctypes.data] * 3
    fn = getattr(L, MANGLED)
    fn.argtypes = [ctypes.c_void_p] * 32 + [ctypes.c_int] * 24 + [ctypes.c_void_p] * 3
    fn.restype = None
    fn(*args)
    counts = (ctypes.c_int64 * 64)()
    assert L.cuapss_compat_counts(counts) == 0
    # oracle on the union, partition of every pair
    rp = np.concatenate([[0]] + [p.rowptr[1:] + sum(q.nnz for q in parts[:k])
                                 for k, p in enumerate(parts)])
    x = synth.Csr(rp, np.concatenate([p.col for p in parts]),
                  np.concatenate([p.val for p in parts]), cfg.d)
    i, j, _ = oracle.apss(x, t)
    first = np.concatenate([[0], np.cumsum(sizes)])
    pa = np.searchsorted(first, i, side="right") - 1
    pb = np.searchsorted(first, j, side="right") - 1
    want = np.zeros(64, np.int64)
    np.add.at(want, 8 * np.minimum(pa, pb) + np.maximum(pa, pb), 1)
    np.testing.assert_array_equal(np.array(counts[:]), want)
    assert want.sum() > 0
    text = capfd.readouterr().out
    lines = re.findall(r"par_([A-H]) (?:join par_([A-H])|apss): sum pair=(\d+)", text)
    assert len(lines) == 28 + 8
    for a, b, c in lines:
        x_, y_ = ord(a) - 65, (ord(b) - 65 if b else ord(a) - 65)
        assert int(c) == want[8 * x_ + y_]


# ---- the reference's text input format (main.cu:301-323) ----

def _reference_lines(x, rng):
    """Lines as the reference's loader reads them: one leading separator
    character, then "d v" pairs each followed by one character (a separator
    or the newline); entries in any order, mixed whitespace inside a pair."""
    out = []
    for r in range(x.n):
        a, b = int(x.rowptr[r]), int(x.rowptr[r + 1])
        if a == b:
            out.append("\n")
            continue
        parts = []
        for e in rng.permutation(np.arange(a, b)):
            gap = " " if rng.uniform() < 0.7 else "\t "
            parts.append(f"{int(x.col[e])}{gap}{float(x.val[e]):.9g}")
        sep = "\t" if r % 3 == 0 else " "
        out.append(sep + sep.join(parts) + "\n")
    return "".join(out)


def test_text_format_reads_reference_lines(tmp_path):
    x = synth.generate("plain_20k", n=300)
    # a few empty vectors, as an empty line
    rp = x.rowptr.copy()
    keep = np.ones(x.n, bool)
    keep[[5, 77, 299]] = False
    lens = np.where(keep, np.diff(rp), 0)
    idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in range(x.n) if keep[r]])
    y = synth.Csr(np.concatenate([[0], np.cumsum(lens)]), x.col[idx], x.val[idx], x.d)
    p = tmp_path / "vectors.txt"
    p.write_text(_reference_lines(y, np.random.default_rng(1)))
    z = cuapss.read_text(str(p))
    assert z.n == y.n and z.d == int(y.col.max()) + 1
    np.testing.assert_array_equal(z.rowptr, y.rowptr)
    np.testing.assert_array_equal(z.col, y.col)
    np.testing.assert_array_equal(z.val, y.val)
    # the first rows only
    w = cuapss.read_text(str(p), max_rows=10)
    assert w.n == 10 and w.nnz == int(y.rowptr[10])


def test_text_format_round_trip_through_tile_ell(tmp_path):
    x = synth.generate("plain_20k", n=517)
    p = tmp_path / "x.txt"
    cuapss.write_text(str(p), x)
    y = cuapss.read_text(str(p))
    np.testing.assert_array_equal(y.rowptr, x.rowptr)
    np.testing.assert_array_equal(y.col, x.col)
    np.testing.assert_array_equal(y.val, x.val)
    # the reference builds its tile-ELL partitions from these vectors
    dim, feat, ts = to_tile_ell(y, np.random.default_rng(2))
    m, rp, col, val = convert(dim, feat, ts, y.n)
    assert m == x.nnz
    np.testing.assert_array_equal(rp, x.rowptr)
    np.testing.assert_array_equal(col, x.col)
    np.testing.assert_array_equal(val, x.val)


@pytest.mark.parametrize("bad", [" 3 0.5 3 0.25\n",       # id repeated in a vector
                                 " 3 0.5 -2 0.25\n",      # negative id
                                 " 3 0.5 x 0.25\n",       # not a number
                                 " 3 0.5 7\n"])           # missing value
def test_text_format_rejects_malformed(tmp_path, bad):
    p = tmp_path / "bad.txt"
    p.write_text(" 1 0.5 2 0.5\n" + bad)
    with pytest.raises(ValueError):
        cuapss.read_text(str(p))
    assert cuapss.read_text(str(p), max_rows=1).n == 1
    with pytest.raises(ValueError):
        cuapss.read_text(str(tmp_path / "missing.txt"))
