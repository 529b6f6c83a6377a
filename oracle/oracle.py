"""ctypes binding of the CPU oracle (oracle.c) -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
the product path (apss-cuda_b200/) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_p = ctypes.c_void_p
_i64 = ctypes.c_int64


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "lib", "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_apss_fp64.argtypes = [_i64, _i64, _p, _p, _p, ctypes.c_double, _i64, _p, _p, _p]
        L.oracle_apss_fp64.restype = _i64
        L.oracle_join_fp64.argtypes = [_i64, _p, _p, _p, _i64, _p, _p, _p, _i64,
                                       ctypes.c_double, _i64, _p, _p, _p]
        L.oracle_join_fp64.restype = _i64
        L.oracle_pair_sims.argtypes = [_p, _p, _p, _i64, _p, _p, _p]
        L.oracle_pair_sims.restype = None
        L.oracle_rows_fp64.argtypes = [_i64, _i64, _p, _p, _p, ctypes.c_double, _i64, _p,
                                       _i64, _p, _p, _p]
        L.oracle_rows_fp64.restype = _i64
        L.oracle_index_ref.argtypes = [_i64, _i64, _p, _p, _p, ctypes.c_int32, _p, _p, _p]
        L.oracle_index_ref.restype = _i64
        L.oracle_feature_remap.argtypes = [_i64, _i64, _p, _p, _p, _p]
        L.oracle_feature_remap.restype = None
        L.cpu_hybrid_apss.argtypes = [_i64, _i64, _p, _p, _p, ctypes.c_float, ctypes.c_int32,
                                      _i64, _i64, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double)]
        L.cpu_hybrid_apss.restype = _i64
        L.cpu_hybrid_prepare.argtypes = [_i64, _i64, _p, _p, _p, ctypes.c_int32, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]
        L.cpu_hybrid_prepare.restype = ctypes.c_void_p
        L.cpu_hybrid_query.argtypes = [ctypes.c_void_p, ctypes.c_float, _i64, _p, _i64,
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.cpu_hybrid_query.restype = _i64
        L.cpu_hybrid_free.argtypes = [ctypes.c_void_p]
        L.cpu_hybrid_free.restype = None
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _call_pairs(fn, args, cap_guess):
    cap = max(cap_guess, 16)
    while True:
        oi = np.empty(cap, np.int32)
        oj = np.empty(cap, np.int32)
        os_ = np.empty(cap, np.float64)
        total = fn(*args, cap, oi.ctypes.data, oj.ctypes.data, os_.ctypes.data)
        if total < 0:
            raise ValueError("oracle rejected the input")
        if total <= cap:
            return oi[:total], oj[:total], os_[:total]
        cap = int(total)


def apss(x, t: float):
    """All pairs i < j with FP64 similarity >= t, sorted by (i, j)."""
    return _call_pairs(lib().oracle_apss_fp64,
                       (x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data, x.val.ctypes.data,
                        float(t)), 1 << 16)


def join(a, b, t: float):
    d = max(a.d, b.d)
    return _call_pairs(lib().oracle_join_fp64,
                       (a.n, a.rowptr.ctypes.data, a.col.ctypes.data, a.val.ctypes.data,
                        b.n, b.rowptr.ctypes.data, b.col.ctypes.data, b.val.ctypes.data,
                        d, float(t)), 1 << 16)


def rows(x, t: float, rows_):
    r = np.ascontiguousarray(rows_, dtype=np.int32)
    return _call_pairs(lib().oracle_rows_fp64,
                       (x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data, x.val.ctypes.data,
                        float(t), len(r), r.ctypes.data), 1 << 16)


def pair_sims(x, pi, pj):
    pi = np.ascontiguousarray(pi, dtype=np.int32)
    pj = np.ascontiguousarray(pj, dtype=np.int32)
    out = np.empty(len(pi), np.float64)
    lib().oracle_pair_sims(x.rowptr.ctypes.data, x.col.ctypes.data, x.val.ctypes.data,
                           len(pi), pi.ctypes.data, pj.ctypes.data, out.ctypes.data)
    return out


def index_ref(x, p: int):
    """(dim_ptr[d+1] int32, rows int32, vals float32) of the reference index."""
    dim_ptr = np.empty(x.d + 1, np.int32)
    cap = max(int((x.col >= p).sum()), 1)
    rows_ = np.empty(cap, np.int32)
    vals = np.empty(cap, np.float32)
    tot = lib().oracle_index_ref(x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data,
                                 x.val.ctypes.data, int(p), dim_ptr.ctypes.data,
                                 rows_.ctypes.data, vals.ctypes.data)
    if tot < 0:
        raise ValueError("oracle rejected the input")
    return dim_ptr, rows_[:tot], vals[:tot]


def feature_remap(x):
    perm = np.empty(x.d, np.int32)
    counts = np.empty(x.d, np.int32)
    lib().oracle_feature_remap(x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data,
                               perm.ctypes.data, counts.ctypes.data)
    return perm, counts


def cpu_hybrid(x, t: float, p: int, q0: int, q1: int, threads: int = 0):
    """(count, prep seconds, query seconds) of the OpenMP FP32 hybrid."""
    sp = ctypes.c_double()
    sq = ctypes.c_double()
    c = lib().cpu_hybrid_apss(x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data,
                              x.val.ctypes.data, float(t), int(p), int(q0), int(q1),
                              int(threads), ctypes.byref(sp), ctypes.byref(sq))
    if c < 0:
        raise ValueError("cpu_hybrid rejected the input")
    return int(c), sp.value, sq.value


class CpuHybrid:
    """The OpenMP FP32 hybrid with its preprocessing done once: prep_s holds
    its wall seconds; query(t, rows) counts the pairs (i, j > i) of the given
    query rows and returns (count, seconds)."""

    def __init__(self, x, p: int, threads: int = 0):
        self._x = x  # the handle points into x's arrays
        self.threads = int(threads)
        sp = ctypes.c_double()
        self._h = lib().cpu_hybrid_prepare(x.n, x.d, x.rowptr.ctypes.data, x.col.ctypes.data,
                                           x.val.ctypes.data, int(p), self.threads,
                                           ctypes.byref(sp))
        if not self._h:
            raise ValueError("cpu_hybrid_prepare rejected the input")
        self.prep_s = sp.value

    def query(self, t: float, rows):
        r = np.ascontiguousarray(rows, dtype=np.int64)
        sq = ctypes.c_double()
        c = lib().cpu_hybrid_query(self._h, float(t), len(r), r.ctypes.data, 0, self.threads,
                                   ctypes.byref(sq))
        if c < 0:
            raise ValueError("cpu_hybrid_query failed")
        return int(c), sq.value

    def close(self):
        if self._h:
            lib().cpu_hybrid_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def ref_cpu_search_path():
    p = os.path.join(HERE, "_ref", "ref_cpu_search")
    return p if os.path.exists(p) else None


def ref_index_path():
    p = os.path.join(HERE, "_ref", "ref_index")
    return p if os.path.exists(p) else None
