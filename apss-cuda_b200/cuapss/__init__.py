"""Python host binding of the CuAPSS C ABI (include/cuapss.h).

Mirrors the reference's one entry point -- similarity_join_device
(fengyilin118/APSS-CUDA similarity_search.h:3-14), which takes the
pre-processed vectors and reports the pairs whose cosine similarity is >= the
threshold -- as a context object with ``run`` (self-join), ``join``
(cross-join), ``build_index`` (the reference's inverted index) and
``feature_remap``. All compute happens in ``lib/libcuapss.so``; if the
library is missing this module raises instead of falling back to anything.

Inputs are :class:`cuapss.synth.Csr` host matrices (numpy) or dictionaries
of CUDA torch tensors ``{"rowptr", "col", "val", "d"}`` (device pointers are
then passed straight through).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .synth import Csr, CONFIGS, SynthConfig, generate  # noqa: F401

_LIB_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib")
LIB_PATH = os.path.join(_LIB_DIR, "libcuapss.so")

OK, EINVAL, ENOMEM, EOVERFLOW, ETIMEOUT, ECUDA, EBUSY = range(7)
PREC_FP32, PREC_MIXED = 0, 1


class CuapssError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


class Opts(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("precision", ctypes.c_int),
        ("head_width", ctypes.c_int),
        ("remap", ctypes.c_int),
        ("validate", ctypes.c_int),
        ("norm_tol", ctypes.c_float),
        ("verbose", ctypes.c_int),
        ("rare_max_count", ctypes.c_int),
    ]


class CsrDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64),
        ("d", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
        ("rowptr", ctypes.c_void_p),
        ("col", ctypes.c_void_p),
        ("val", ctypes.c_void_p),
        ("on_device", ctypes.c_int),
    ]


class PairsDesc(ctypes.Structure):
    _fields_ = [
        ("i", ctypes.c_void_p),
        ("j", ctypes.c_void_p),
        ("sim", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("count", ctypes.c_int64),
        ("on_device", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("pairs", ctypes.c_int64),
        ("candidates", ctypes.c_int64),
        ("rescored", ctypes.c_int64),
        ("tiles", ctypes.c_int64),
        ("head_width", ctypes.c_int64),
        ("tail_entries", ctypes.c_int64),
        ("tail_products", ctypes.c_int64),
        ("max_band", ctypes.c_double),
        ("ms_preprocess", ctypes.c_double),
        ("ms_index", ctypes.c_double),
        ("ms_tiles", ctypes.c_double),
        ("ms_finalize", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("launches", ctypes.c_int64),
        ("explicit_pairs", ctypes.c_int64),
        ("rare_max_count", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.c_void_p
_lib = None

# Every symbol declared by include/cuapss.h (checked by the CPU tests).
class ServerOpts(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_int32), ("max_batch_rows", ctypes.c_int64),
                ("hbm_budget", ctypes.c_int64)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("pairs", ctypes.c_int64),
                ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("batch_id", ctypes.c_int64), ("batch_rows", ctypes.c_int64),
                ("index_rows", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


EXPORTED = [
    "cuapss_default_opts", "cuapss_status_string", "cuapss_abi_version", "cuapss_create",
    "cuapss_destroy", "cuapss_run", "cuapss_join", "cuapss_build_index", "cuapss_feature_remap",
    "cuapss_batch_run", "cuapss_selftest_bounded_wait", "cuapss_run_shard", "cuapss_shard_blocks", "cuapss_index_create", "cuapss_index_append", "cuapss_index_query",
    "cuapss_index_info", "cuapss_index_destroy", "cuapss_server_default_opts",
    "cuapss_server_create", "cuapss_server_submit_query", "cuapss_server_submit_append",
    "cuapss_server_wait", "cuapss_server_destroy",
]


def lib():
    """Load lib/libcuapss.so (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        L.cuapss_default_opts.argtypes = [ctypes.POINTER(Opts)]
        L.cuapss_default_opts.restype = None
        L.cuapss_status_string.argtypes = [ctypes.c_int]
        L.cuapss_status_string.restype = ctypes.c_char_p
        L.cuapss_abi_version.restype = ctypes.c_int
        L.cuapss_create.argtypes = [ctypes.POINTER(_P), ctypes.POINTER(Opts)]
        L.cuapss_create.restype = ctypes.c_int
        L.cuapss_destroy.argtypes = [_P]
        L.cuapss_destroy.restype = ctypes.c_int
        L.cuapss_run.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.c_float,
                                 ctypes.POINTER(PairsDesc), ctypes.POINTER(Stats)]
        L.cuapss_run.restype = ctypes.c_int
        L.cuapss_join.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.POINTER(CsrDesc),
                                  ctypes.c_float, ctypes.POINTER(PairsDesc),
                                  ctypes.POINTER(Stats)]
        L.cuapss_join.restype = ctypes.c_int
        L.cuapss_build_index.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.c_int32, _P, _P, _P,
                                         ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.cuapss_build_index.restype = ctypes.c_int
        L.cuapss_feature_remap.argtypes = [_P, ctypes.POINTER(CsrDesc), _P, _P]
        L.cuapss_feature_remap.restype = ctypes.c_int
        L.cuapss_batch_run.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.c_int32, _P, _P,
                                       ctypes.POINTER(PairsDesc), ctypes.POINTER(Stats), _P]
        L.cuapss_batch_run.restype = ctypes.c_int
        L.cuapss_selftest_bounded_wait.argtypes = [_P, ctypes.c_int32,
                                                   ctypes.POINTER(ctypes.c_int64)]
        L.cuapss_selftest_bounded_wait.restype = ctypes.c_int
        L.cuapss_run_shard.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.c_float, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.POINTER(PairsDesc),
                                       ctypes.POINTER(Stats)]
        L.cuapss_run_shard.restype = ctypes.c_int
        L.cuapss_shard_blocks.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P,
                                          ctypes.c_int64]
        L.cuapss_shard_blocks.restype = ctypes.c_int32
        L.cuapss_plan_self_join.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, _P,
                                            ctypes.c_int64, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int64)]
        L.cuapss_plan_self_join.restype = ctypes.c_int
        L.cuapss_index_create.argtypes = [_P, ctypes.POINTER(CsrDesc), ctypes.POINTER(_P)]
        L.cuapss_index_create.restype = ctypes.c_int
        L.cuapss_index_append.argtypes = [_P, _P, ctypes.POINTER(CsrDesc)]
        L.cuapss_index_append.restype = ctypes.c_int
        L.cuapss_index_query.argtypes = [_P, _P, ctypes.POINTER(CsrDesc), _P,
                                         ctypes.POINTER(PairsDesc), ctypes.POINTER(Stats)]
        L.cuapss_index_query.restype = ctypes.c_int
        L.cuapss_index_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_int64)]
        L.cuapss_index_info.restype = ctypes.c_int
        L.cuapss_index_destroy.argtypes = [_P]
        L.cuapss_index_destroy.restype = ctypes.c_int
        L.cuapss_server_default_opts.argtypes = [ctypes.POINTER(ServerOpts)]
        L.cuapss_server_default_opts.restype = None
        L.cuapss_server_create.argtypes = [ctypes.POINTER(_P), _P, ctypes.c_int,
                                           ctypes.POINTER(ServerOpts)]
        L.cuapss_server_create.restype = ctypes.c_int
        L.cuapss_server_submit_query.argtypes = [_P, ctypes.POINTER(CsrDesc), _P,
                                                 ctypes.POINTER(ctypes.c_uint64)]
        L.cuapss_server_submit_query.restype = ctypes.c_int
        L.cuapss_server_submit_append.argtypes = [_P, ctypes.POINTER(CsrDesc),
                                                  ctypes.POINTER(ctypes.c_uint64)]
        L.cuapss_server_submit_append.restype = ctypes.c_int
        L.cuapss_server_wait.argtypes = [_P, ctypes.c_uint64, ctypes.c_int32,
                                         ctypes.POINTER(PairsDesc), ctypes.POINTER(RequestInfo)]
        L.cuapss_server_wait.restype = ctypes.c_int
        L.cuapss_server_destroy.argtypes = [_P]
        L.cuapss_server_destroy.restype = ctypes.c_int
        _lib = L
    return _lib


def status_string(s: int) -> str:
    return lib().cuapss_status_string(int(s)).decode()


def default_opts() -> Opts:
    o = Opts()
    lib().cuapss_default_opts(ctypes.byref(o))
    return o


def _check(status: int, what: str) -> None:
    if status != OK:
        raise CuapssError(status, what)


def _desc(x) -> tuple:
    """(CsrDesc, keepalive) for a host Csr or a dict of CUDA tensors."""
    if isinstance(x, Csr):
        d = CsrDesc(x.n, x.d, x.nnz, x.rowptr.ctypes.data, x.col.ctypes.data,
                    x.val.ctypes.data, 0)
        return d, x
    rp, col, val = x["rowptr"], x["col"], x["val"]
    d = CsrDesc(int(rp.numel()) - 1, int(x["d"]), int(col.numel()), rp.data_ptr(),
                col.data_ptr(), val.data_ptr(), 1)
    return d, x


class Context:
    """One CuAPSS context (one device, one stream, one host thread at a time)."""

    def __init__(self, device: int = 0, precision: int = PREC_FP32, head_width: int = 0,
                 remap: bool = True, validate: bool = True, norm_tol: float = 1e-4,
                 stream: int | None = None, rare_max_count: int = 0):
        o = default_opts()
        o.device = device
        o.precision = precision
        o.head_width = head_width
        o.remap = 1 if remap else 0
        o.validate = 1 if validate else 0
        o.norm_tol = norm_tol
        o.stream = stream
        o.rare_max_count = rare_max_count
        self._h = _P()
        _check(lib().cuapss_create(ctypes.byref(self._h), ctypes.byref(o)), "cuapss_create")
        self.last_stats: dict = {}

    def close(self) -> None:
        if self._h:
            lib().cuapss_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _pairs_call(self, fn, args, capacity: int):
        cap = max(int(capacity), 1)
        while True:
            oi = np.empty(cap, np.int32)
            oj = np.empty(cap, np.int32)
            os_ = np.empty(cap, np.float32)
            pr = PairsDesc(oi.ctypes.data, oj.ctypes.data, os_.ctypes.data, cap, 0, 0)
            st = Stats()
            s = fn(self._h, *args, ctypes.byref(pr), ctypes.byref(st))
            if s == EOVERFLOW:
                cap = int(pr.count)
                continue
            _check(s, fn.__name__)
            self.last_stats = st.as_dict()
            n = int(pr.count)
            return oi[:n].copy(), oj[:n].copy(), os_[:n].copy()

    def run(self, x, t: float, capacity: int = 1 << 16):
        """Self-join: (i, j, sim) numpy arrays, i < j, sorted by (i, j)."""
        d, keep = _desc(x)
        return self._pairs_call(lib().cuapss_run, (ctypes.byref(d), ctypes.c_float(t)), capacity)

    def selftest_bounded_wait(self, limit_us: int = 1000):
        """(status, device ns waited) of the bounded-wait self-check with a
        deadline of limit_us; the expected status is ETIMEOUT."""
        waited = ctypes.c_int64()
        s = lib().cuapss_selftest_bounded_wait(self._h, int(limit_us), ctypes.byref(waited))
        return s, waited.value

    def run_shard(self, x, t: float, shard: int, nshards: int, capacity: int = 1 << 16):
        """One shard of run(): pairs whose row i lies in a 128-row block b with
        b % nshards == shard; the shards' union is run()'s output."""
        d, keep = _desc(x)
        return self._pairs_call(lib().cuapss_run_shard,
                                (ctypes.byref(d), ctypes.c_float(t), int(shard), int(nshards)),
                                capacity)

    def run_shard_device(self, x, t: float, shard: int, nshards: int, out: dict):
        """run_shard into CUDA tensors out = {"i", "j", "sim"}; returns the
        pair count (raises CuapssError(EOVERFLOW) with self.required set)."""
        d, keep = _desc(x)
        cap = int(out["i"].numel())
        pr = PairsDesc(out["i"].data_ptr(), out["j"].data_ptr(), out["sim"].data_ptr(), cap, 0, 1)
        st = Stats()
        s = lib().cuapss_run_shard(self._h, ctypes.byref(d), ctypes.c_float(t), int(shard),
                                   int(nshards), ctypes.byref(pr), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if s == EOVERFLOW:
            self.required = int(pr.count)
        _check(s, "cuapss_run_shard")
        return int(pr.count)

    def run_device(self, x, t: float, out: dict):
        """Self-join into CUDA tensors out = {"i", "j", "sim"}; returns the
        pair count (raises CuapssError(EOVERFLOW) with .status if short)."""
        d, keep = _desc(x)
        cap = int(out["i"].numel())
        pr = PairsDesc(out["i"].data_ptr(), out["j"].data_ptr(), out["sim"].data_ptr(), cap, 0, 1)
        st = Stats()
        s = lib().cuapss_run(self._h, ctypes.byref(d), ctypes.c_float(t), ctypes.byref(pr),
                             ctypes.byref(st))
        self.last_stats = st.as_dict()
        if s == EOVERFLOW:
            self.required = int(pr.count)
        _check(s, "cuapss_run")
        return int(pr.count)

    def join(self, a, b, t: float, capacity: int = 1 << 16):
        """Cross-join: (i in a, j in b, sim), sorted by (i, j)."""
        da, ka = _desc(a)
        db, kb = _desc(b)
        return self._pairs_call(lib().cuapss_join,
                                (ctypes.byref(da), ctypes.byref(db), ctypes.c_float(t)), capacity)

    def _batch_args(self, x, inst_ptr, t):
        d, keep = _desc(x)
        ip = np.ascontiguousarray(inst_ptr, dtype=np.int64)
        tq = np.ascontiguousarray(t, dtype=np.float32)
        if ip.ndim != 1 or tq.shape != (ip.size - 1,):
            raise ValueError("inst_ptr has k+1 entries and t has k")
        return d, keep, ip, tq

    def batch_run(self, x, inst_ptr, t, capacity: int = 1 << 16):
        """Batched self-joins of the row ranges [inst_ptr[q], inst_ptr[q+1])
        of x, instance q at threshold t[q]: (i, j, sim) in x's rows, sorted.
        The head width used per size bucket is left in self.last_bucket_p."""
        d, keep, ip, tq = self._batch_args(x, inst_ptr, t)
        cap = max(int(capacity), 1)
        bp = np.zeros(3, np.int32)
        while True:
            oi = np.empty(cap, np.int32)
            oj = np.empty(cap, np.int32)
            os_ = np.empty(cap, np.float32)
            pr = PairsDesc(oi.ctypes.data, oj.ctypes.data, os_.ctypes.data, cap, 0, 0)
            st = Stats()
            s = lib().cuapss_batch_run(self._h, ctypes.byref(d), int(tq.size), ip.ctypes.data,
                                       tq.ctypes.data, ctypes.byref(pr), ctypes.byref(st),
                                       bp.ctypes.data)
            if s == EOVERFLOW:
                cap = int(pr.count)
                continue
            _check(s, "cuapss_batch_run")
            self.last_stats = st.as_dict()
            self.last_bucket_p = bp.copy()
            n = int(pr.count)
            return oi[:n].copy(), oj[:n].copy(), os_[:n].copy()

    def batch_run_device(self, x, inst_ptr, t, out: dict):
        """batch_run with x a dict of CUDA tensors and the pairs written to
        CUDA tensors out = {"i", "j", "sim"}; returns the pair count (raises
        CuapssError(EOVERFLOW) with self.required set if short)."""
        d, keep, ip, tq = self._batch_args(x, inst_ptr, t)
        cap = int(out["i"].numel())
        pr = PairsDesc(out["i"].data_ptr(), out["j"].data_ptr(), out["sim"].data_ptr(), cap, 0, 1)
        st = Stats()
        bp = np.zeros(3, np.int32)
        s = lib().cuapss_batch_run(self._h, ctypes.byref(d), int(tq.size), ip.ctypes.data,
                                   tq.ctypes.data, ctypes.byref(pr), ctypes.byref(st),
                                   bp.ctypes.data)
        self.last_stats = st.as_dict()
        self.last_bucket_p = bp.copy()
        if s == EOVERFLOW:
            self.required = int(pr.count)
        _check(s, "cuapss_batch_run")
        return int(pr.count)

    def build_index(self, x: Csr, p: int):
        """Reference-semantics tail index: (dim_ptr[d+1], rows, vals)."""
        d, keep = _desc(x)
        dim_ptr = np.empty(x.d + 1, np.int32)
        cap = max(int((x.col >= p).sum()), 1)
        rows = np.empty(cap, np.int32)
        vals = np.empty(cap, np.float32)
        tn = ctypes.c_int64()
        _check(lib().cuapss_build_index(self._h, ctypes.byref(d), int(p), dim_ptr.ctypes.data,
                                        rows.ctypes.data, vals.ctypes.data, cap,
                                        ctypes.byref(tn)), "cuapss_build_index")
        return dim_ptr, rows[:tn.value], vals[:tn.value]

    def feature_remap(self, x: Csr):
        d, keep = _desc(x)
        perm = np.empty(x.d, np.int32)
        counts = np.empty(x.d, np.int32)
        _check(lib().cuapss_feature_remap(self._h, ctypes.byref(d), perm.ctypes.data,
                                          counts.ctypes.data), "cuapss_feature_remap")
        return perm, counts


class Index:
    """Resident index (cuapss_index_*): rows kept in HBM for repeated query
    batches with per-query thresholds; appends add rows."""

    def __init__(self, ctx: "Context", x):
        self.ctx = ctx
        self._h = _P()
        d, keep = _desc(x)
        _check(lib().cuapss_index_create(ctx._h, ctypes.byref(d), ctypes.byref(self._h)),
               "cuapss_index_create")

    def append(self, x, ctx: "Context | None" = None):
        d, keep = _desc(x)
        c = ctx or self.ctx
        _check(lib().cuapss_index_append(c._h, self._h, ctypes.byref(d)), "cuapss_index_append")

    def info(self) -> dict:
        r, s, p, b = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        _check(lib().cuapss_index_info(self._h, ctypes.byref(r), ctypes.byref(s), ctypes.byref(p),
                                       ctypes.byref(b)), "cuapss_index_info")
        return {"rows": r.value, "segments": s.value, "head_width": p.value,
                "device_bytes": b.value}

    def query(self, q, t, capacity: int = 1 << 16, ctx: "Context | None" = None):
        """(i = query row, j = index row, sim), sorted by (i, j); t is one
        threshold or one per query row."""
        c = ctx or self.ctx
        d, keep = _desc(q)
        tq = np.ascontiguousarray(np.broadcast_to(np.asarray(t, np.float32), (d.n,)))
        cap = max(int(capacity), 1)
        while True:
            oi = np.empty(cap, np.int32)
            oj = np.empty(cap, np.int32)
            os_ = np.empty(cap, np.float32)
            pr = PairsDesc(oi.ctypes.data, oj.ctypes.data, os_.ctypes.data, cap, 0, 0)
            st = Stats()
            s = lib().cuapss_index_query(c._h, self._h, ctypes.byref(d), tq.ctypes.data,
                                         ctypes.byref(pr), ctypes.byref(st))
            if s == EOVERFLOW:
                cap = int(pr.count)
                continue
            _check(s, "cuapss_index_query")
            c.last_stats = st.as_dict()
            n = int(pr.count)
            return oi[:n].copy(), oj[:n].copy(), os_[:n].copy()

    def close(self):
        if self._h:
            lib().cuapss_index_destroy(self._h)
            self._h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request server over an Index (cuapss_server_*): continuous batching
    of query requests on several lanes, ordered appends."""

    def __init__(self, index: "Index", device: int = 0, lanes: int = 3,
                 max_batch_rows: int = 1024, hbm_budget: int = 16 << 30):
        o = ServerOpts()
        lib().cuapss_server_default_opts(ctypes.byref(o))
        o.lanes, o.max_batch_rows, o.hbm_budget = lanes, max_batch_rows, hbm_budget
        self.index = index
        self._h = _P()
        _check(lib().cuapss_server_create(ctypes.byref(self._h), index._h, device,
                                          ctypes.byref(o)), "cuapss_server_create")

    def submit_query(self, q: Csr, t) -> int:
        d, keep = _desc(q)
        tq = np.ascontiguousarray(np.broadcast_to(np.asarray(t, np.float32), (d.n,)))
        tk = ctypes.c_uint64()
        _check(lib().cuapss_server_submit_query(self._h, ctypes.byref(d), tq.ctypes.data,
                                                ctypes.byref(tk)), "cuapss_server_submit_query")
        return tk.value

    def submit_append(self, x: Csr) -> int:
        d, keep = _desc(x)
        tk = ctypes.c_uint64()
        _check(lib().cuapss_server_submit_append(self._h, ctypes.byref(d), ctypes.byref(tk)),
               "cuapss_server_submit_append")
        return tk.value

    def wait(self, ticket: int, timeout_ms: int = -1, capacity: int = 1 << 16):
        """((i, j, sim), info) of a request; i numbered within the request."""
        cap = max(int(capacity), 1)
        while True:
            oi = np.empty(cap, np.int32)
            oj = np.empty(cap, np.int32)
            os_ = np.empty(cap, np.float32)
            pr = PairsDesc(oi.ctypes.data, oj.ctypes.data, os_.ctypes.data, cap, 0, 0)
            info = RequestInfo()
            s = lib().cuapss_server_wait(self._h, int(ticket), int(timeout_ms), ctypes.byref(pr),
                                         ctypes.byref(info))
            if s == EOVERFLOW:
                cap = int(pr.count)
                continue
            _check(s, "cuapss_server_wait")
            n = int(pr.count)
            return (oi[:n].copy(), oj[:n].copy(), os_[:n].copy()), info.as_dict()

    def close(self):
        if self._h:
            lib().cuapss_server_destroy(self._h)
            self._h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_self_join(x, precision: int = PREC_MIXED, max_pairs: int = 0) -> dict:
    """The plan cuapss_run makes for a self-join of x (a Csr, or a pair
    (posting counts per feature, n rows)), computed on the host: head width,
    rare-feature threshold (0: none) and the explicit pairs it implies."""
    if isinstance(x, tuple):
        counts, n = x
        counts = np.ascontiguousarray(counts, dtype=np.int32)
    else:
        counts = np.bincount(x.col, minlength=x.d).astype(np.int32)
        n = x.n
    p = ctypes.c_int32()
    c = ctypes.c_int32()
    pairs = ctypes.c_int64()
    _check(lib().cuapss_plan_self_join(int(precision), int(n), len(counts), counts.ctypes.data,
                                       int(max_pairs), ctypes.byref(p), ctypes.byref(c),
                                       ctypes.byref(pairs)), "cuapss_plan_self_join")
    return {"head_width": p.value, "rare_max_count": c.value, "explicit_pairs": pairs.value}


def shard_blocks(n: int, shard: int, nshards: int) -> np.ndarray:
    """Row blocks (128 rows each) of an n-row self-join owned by a shard."""
    m = lib().cuapss_shard_blocks(int(n), int(shard), int(nshards), None, 0)
    if m < 0:
        raise ValueError("bad shard arguments")
    out = np.empty(max(m, 1), np.int32)
    lib().cuapss_shard_blocks(int(n), int(shard), int(nshards), out.ctypes.data, m)
    return out[:m]


def read_text(path: str, max_rows: int = -1) -> Csr:
    """Vectors of a file in the reference's text format (one vector per line,
    "d v" pairs; main.cu:301-323) as a CSR matrix, rows sorted by feature id,
    d = largest id + 1 (cuapss_compat_read_text)."""
    L = lib()
    f = L.cuapss_compat_text_size
    f.argtypes = [ctypes.c_char_p, ctypes.c_int64] + [ctypes.POINTER(ctypes.c_int64)] * 3
    f.restype = ctypes.c_int
    n, nnz, d = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    if f(os.fsencode(path), int(max_rows), ctypes.byref(n), ctypes.byref(nnz),
         ctypes.byref(d)) != 0:
        raise ValueError(f"{path}: not in the reference's text format")
    g = L.cuapss_compat_read_text
    g.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    g.restype = ctypes.c_int
    rp = np.zeros(n.value + 1, np.int64)
    col = np.empty(max(nnz.value, 1), np.int32)
    val = np.empty(max(nnz.value, 1), np.float32)
    if g(os.fsencode(path), int(max_rows), rp.ctypes.data, col.ctypes.data,
         val.ctypes.data) != 0:
        raise ValueError(f"{path}: not in the reference's text format")
    return Csr(rp, col[:nnz.value], val[:nnz.value], max(d.value, 1))


def write_text(path: str, x) -> None:
    """Writes x in the reference's text format (cuapss_compat_write_text)."""
    f = lib().cuapss_compat_write_text
    f.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    if f(os.fsencode(path), x.n, x.rowptr.ctypes.data, x.col.ctypes.data,
         x.val.ctypes.data) != 0:
        raise OSError(f"cannot write {path}")
