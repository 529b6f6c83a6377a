"""C-ABI library checks that need no GPU: it loads, exports every function
include/*.h declares, and rejects calls cleanly without a device."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import cuapss
from cuapss import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cuapss_[a-z0-9_]+)\s*\(", src)))


def _exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_every_declared_symbol_is_exported():
    names = _declared("cuapss.h")
    assert "cuapss_run" in names and "cuapss_build_index" in names
    exp = _exported(cuapss.LIB_PATH)
    missing = [n for n in names if n not in exp]
    assert not missing, missing
    assert set(cuapss.EXPORTED) <= exp


def test_every_compat_symbol_is_exported():
    names = _declared("cuapss_compat.h")
    assert "cuapss_compat_read_text" in names
    exp = _exported(cuapss.LIB_PATH)
    missing = [n for n in names if n not in exp]
    assert not missing, missing


def test_synth_symbols_exported():
    exp = _exported(os.path.join(ROOT, "apss-cuda_b200", "lib", "libcuapss_synth.so"))
    for n in _declared("cuapss_synth.h"):
        assert n in exp


def test_status_strings_and_defaults():
    assert cuapss.lib().cuapss_abi_version() == 2
    assert cuapss.status_string(cuapss.OK) == "ok"
    assert "capacity" in cuapss.status_string(cuapss.EOVERFLOW)
    o = cuapss.default_opts()
    assert o.remap == 1 and o.validate == 1 and o.precision == cuapss.PREC_FP32
    assert abs(o.norm_tol - 1e-4) < 1e-9
    assert o.rare_max_count == 0


def test_create_without_device_fails_cleanly():
    from tests.conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    s = cuapss.lib().cuapss_create(ctypes.byref(h), None)
    assert s in (cuapss.ECUDA, cuapss.EINVAL)
    assert not h.value


def test_bad_options_rejected():
    h = ctypes.c_void_p()
    o = cuapss.default_opts()
    o.precision = 7
    assert cuapss.lib().cuapss_create(ctypes.byref(h), ctypes.byref(o)) == cuapss.EINVAL
    assert cuapss.lib().cuapss_create(None, None) == cuapss.EINVAL
    # the rare-feature threshold: -1, 0 or a power of two in 16 .. 2048
    for bad in (-2, 8, 24, 4096):
        o = cuapss.default_opts()
        o.rare_max_count = bad
        assert cuapss.lib().cuapss_create(ctypes.byref(h), ctypes.byref(o)) == cuapss.EINVAL


def test_synth_determinism_and_shape():
    a = synth.generate("plain_20k", n=3000)
    b = synth.generate("plain_20k", n=3000)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.val, b.val)
    lens = np.diff(a.rowptr)
    assert lens.min() >= 1 and lens.max() <= 500
    for i in range(0, a.n, 101):
        c = a.col[a.rowptr[i]:a.rowptr[i + 1]]
        assert np.all(np.diff(c) > 0) and c.min() >= 0 and c.max() < a.d
    nr = np.sqrt(np.add.reduceat(a.val.astype(np.float64) ** 2, a.rowptr[:-1]))
    assert np.max(np.abs(nr - 1)) < 1e-6
    # rows are a prefix of a longer stream: same seed, same rows
    c = synth.generate("plain_20k", n=1000)
    assert np.array_equal(c.col, a.col[:c.nnz])
    # offset streams continue it
    d = synth.generate("plain_20k", n=500, row_offset=1000)
    assert np.array_equal(d.col, a.col[a.rowptr[1000]:a.rowptr[1500]])


def test_synth_distribution_moments():
    x = synth.generate("plain_800k", n=20000)
    lens = np.diff(x.rowptr)
    assert 60 < lens.mean() < 90  # lognormal mean 75, clipped at 3000
    counts = np.bincount(x.col, minlength=x.d)
    top = np.sort(counts)[::-1]
    assert top[0] > 0.8 * x.n  # the most frequent Zipf(1.1) feature is in most rows
    assert top[1000] < top[10]
