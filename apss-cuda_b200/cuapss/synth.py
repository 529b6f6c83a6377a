"""Seeded synthetic inputs for the APSS benchmark configurations.

Thin ctypes binding of ``lib/libcuapss_synth.so`` (``include/cuapss_synth.h``).
The reference's own corpus (a pre-processed text file read at main.cu:270 of
fengyilin118/APSS-CUDA) is not distributed; these generators stand in for it
with the shapes and distributions of the configurations below.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

_LIB_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib")


class _Params(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64),
        ("d", ctypes.c_int64),
        ("nnz_mean", ctypes.c_double),
        ("nnz_sigma", ctypes.c_double),
        ("nnz_max", ctypes.c_int64),
        ("zipf_s", ctypes.c_double),
        ("tf_p", ctypes.c_double),
        ("dup_frac", ctypes.c_double),
        ("dup_drop", ctypes.c_double),
        ("dup_scale_lo", ctypes.c_double),
        ("dup_scale_hi", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("row_offset", ctypes.c_int64),
        ("stream", ctypes.c_uint64),
    ]


@dataclasses.dataclass(frozen=True)
class SynthConfig:
    """Generator parameters (see include/cuapss_synth.h)."""

    n: int
    d: int
    nnz_mean: float
    nnz_sigma: float
    nnz_max: int
    zipf_s: float
    dup_frac: float
    tf_p: float = 0.3
    dup_drop: float = 0.1
    dup_scale_lo: float = 0.9
    dup_scale_hi: float = 1.1
    seed: int = 0
    stream: int = 0

    def replace(self, **kw) -> "SynthConfig":
        return dataclasses.replace(self, **kw)


# The benchmark configurations (sizes and distributions of the workloads the
# project is measured on).
CONFIGS = {
    # plain hybrid, n=20k, d=10k, lognormal(40, 0.8) clipped 1..500, Zipf 1.0,
    # 5% planted duplicates, t = 0.9
    "plain_20k": SynthConfig(n=20_000, d=10_000, nnz_mean=40, nnz_sigma=0.8,
                             nnz_max=500, zipf_s=1.0, dup_frac=0.05),
    # plain hybrid at scale, n=800k, d=50k, lognormal(75, 1.0) max 3000,
    # Zipf 1.1, 2% duplicates, t in {0.5, 0.7, 0.9}
    "plain_800k": SynthConfig(n=800_000, d=50_000, nnz_mean=75, nnz_sigma=1.0,
                              nnz_max=3000, zipf_s=1.1, dup_frac=0.02),
    # mixed precision, n=1M, d=1M, lognormal(120, 1.0) max 5000, Zipf 1.2
    "mixed_1m": SynthConfig(n=1_000_000, d=1_000_000, nnz_mean=120, nnz_sigma=1.0,
                            nnz_max=5000, zipf_s=1.2, dup_frac=0.02),
    # one instance shape of the batched uneven workload (n varies per instance)
    "batch_instance": SynthConfig(n=1000, d=30_000, nnz_mean=30, nnz_sigma=0.9,
                                  nnz_max=30_000, zipf_s=1.1, dup_frac=0.02),
    # serving: resident index of 5M vectors, d = 2^20, lognormal(60, 1.0)
    "serve_5m": SynthConfig(n=5_000_000, d=1 << 20, nnz_mean=60, nnz_sigma=1.0,
                            nnz_max=5000, zipf_s=1.1, dup_frac=0.02),
}


_lib = None
_lib_path = os.path.join(_LIB_DIR, "libcuapss_synth.so")


def use_library(path: str) -> None:
    """Generate with another build of the same generator source (the CPU
    reference arm of the benchmark uses the copy built under oracle/lib/ so
    that it maps no library of the package). Call before the first
    generate()."""
    global _lib_path
    if _lib is not None and path != _lib_path:
        raise RuntimeError("the generator library is already loaded")
    _lib_path = path


def lib():
    global _lib
    if _lib is None:
        path = _lib_path
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(path)
        L.cuapss_synth_rowptr.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p]
        L.cuapss_synth_rowptr.restype = ctypes.c_int
        L.cuapss_synth_fill.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        L.cuapss_synth_fill.restype = ctypes.c_int
        L.cuapss_synth_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _params(cfg: SynthConfig, row_offset: int = 0) -> _Params:
    return _Params(cfg.n, cfg.d, cfg.nnz_mean, cfg.nnz_sigma, cfg.nnz_max, cfg.zipf_s,
                   cfg.tf_p, cfg.dup_frac, cfg.dup_drop, cfg.dup_scale_lo, cfg.dup_scale_hi,
                   cfg.seed, row_offset, cfg.stream)


class Csr:
    """Host CSR matrix: int64 rowptr[n+1], int32 col[nnz], float32 val[nnz]."""

    def __init__(self, rowptr, col, val, d):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float32)
        self.d = int(d)

    @property
    def n(self) -> int:
        return len(self.rowptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def rows(self, lo: int, hi: int) -> "Csr":
        a, b = int(self.rowptr[lo]), int(self.rowptr[hi])
        return Csr(self.rowptr[lo:hi + 1] - a, self.col[a:b], self.val[a:b], self.d)

    def take(self, rows) -> "Csr":
        rows = np.asarray(rows, dtype=np.int64)
        lens = self.rowptr[rows + 1] - self.rowptr[rows]
        rp = np.zeros(len(rows) + 1, np.int64)
        np.cumsum(lens, out=rp[1:])
        idx = np.concatenate([np.arange(self.rowptr[r], self.rowptr[r + 1]) for r in rows]) \
            if len(rows) else np.zeros(0, np.int64)
        return Csr(rp, self.col[idx], self.val[idx], self.d)

    def save(self, path: str) -> None:
        """Binary layout: int64 n, d, nnz; rowptr; col; val."""
        with open(path, "wb") as f:
            np.array([self.n, self.d, self.nnz], np.int64).tofile(f)
            self.rowptr.tofile(f)
            self.col.tofile(f)
            self.val.tofile(f)

    @staticmethod
    def load(path: str) -> "Csr":
        with open(path, "rb") as f:
            n, d, nnz = np.fromfile(f, np.int64, 3)
            rp = np.fromfile(f, np.int64, n + 1)
            col = np.fromfile(f, np.int32, nnz)
            val = np.fromfile(f, np.float32, nnz)
        return Csr(rp, col, val, d)


def generate(cfg: SynthConfig | str, row_offset: int = 0, **overrides) -> Csr:
    """Generate rows [row_offset, row_offset + n) of the seeded stream."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    if overrides:
        cfg = cfg.replace(**overrides)
    L = lib()
    p = _params(cfg, row_offset)
    rp = np.zeros(cfg.n + 1, np.int64)
    if L.cuapss_synth_rowptr(ctypes.byref(p), rp.ctypes.data) != 0:
        raise ValueError(f"bad generator parameters {cfg}")
    nnz = int(rp[-1])
    col = np.empty(max(nnz, 1), np.int32)
    val = np.empty(max(nnz, 1), np.float32)
    if L.cuapss_synth_fill(ctypes.byref(p), rp.ctypes.data, col.ctypes.data,
                           val.ctypes.data) != 0:
        raise RuntimeError("generator failed")
    return Csr(rp, col[:nnz], val[:nnz], cfg.d)


def host_threads() -> int:
    return int(lib().cuapss_synth_threads())


# The batched workload: 4,096 independent instances, n log-uniform in
# [64, 20,000], thresholds uniform in [0.6, 0.95], rows of "batch_instance".
BATCH = dict(k=4096, n_lo=64, n_hi=20_000, t_lo=0.6, t_hi=0.95)


def generate_batch(k: int = BATCH["k"], n_lo: int = BATCH["n_lo"], n_hi: int = BATCH["n_hi"],
                   t_lo: float = BATCH["t_lo"], t_hi: float = BATCH["t_hi"], seed: int = 0,
                   cfg: SynthConfig | str = "batch_instance"):
    """k independent instances stacked as row ranges of one CSR.

    Instance q has n_q ~ logU[n_lo, n_hi] rows drawn from its own row stream
    (same feature permutation, so the same vocabulary) and threshold
    t_q ~ U[t_lo, t_hi]. Returns (Csr, inst_ptr int64[k+1], t float32[k])."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    rng = np.random.default_rng(seed)
    ns = np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi + 1), size=k))).astype(np.int64)
    ns = np.clip(ns, n_lo, n_hi)
    ts = rng.uniform(t_lo, t_hi, size=k).astype(np.float32)
    inst_ptr = np.zeros(k + 1, np.int64)
    np.cumsum(ns, out=inst_ptr[1:])
    L = lib()
    rp = np.zeros(int(inst_ptr[-1]) + 1, np.int64)
    params = []
    for q in range(k):
        c = cfg.replace(n=int(ns[q]), seed=seed, stream=q + 1)
        pq = _params(c, 0)
        part = np.zeros(int(ns[q]) + 1, np.int64)
        if L.cuapss_synth_rowptr(ctypes.byref(pq), part.ctypes.data) != 0:
            raise ValueError(f"bad generator parameters {c}")
        a = int(inst_ptr[q])
        rp[a + 1:a + 1 + int(ns[q])] = part[1:] + rp[a]
        params.append(pq)
    nnz = int(rp[-1])
    col = np.empty(max(nnz, 1), np.int32)
    val = np.empty(max(nnz, 1), np.float32)
    for q in range(k):
        a, b = int(inst_ptr[q]), int(inst_ptr[q + 1])
        e0 = int(rp[a])
        local = rp[a:b + 1] - e0
        if L.cuapss_synth_fill(ctypes.byref(params[q]), local.ctypes.data,
                               col[e0:].ctypes.data, val[e0:].ctypes.data) != 0:
            raise ValueError("generator failed")
    return Csr(rp, col[:nnz], val[:nnz], cfg.d), inst_ptr, ts
