#!/usr/bin/env python3
"""All-pairs cosine similarity search benchmark (pairs/s).

Workload (default): the hybrid APSS at scale -- n = 800,000 vectors,
d = 50,000, nnz/row lognormal(mean 75, sigma 1.0) clipped at 3,000, Zipf(1.1)
feature ids, tf-log values, 2% planted near-duplicates, threshold t = 0.7,
seeded synthetic data (the reference's corpus is not distributed).

The headline is the mixed-precision path (BF16 head on tcgen05 tensor
cores, FP32 tail, FP64 rescore of the error band -- exact pair set); the
plain FP32 hybrid is timed on the same data and reported beside it.

A step is one complete self-join of that matrix: validate, frequency remap,
row order, head block and inverted lists, all 128 x 128 pair tiles, the exact
finalize and the sorted (i, j, sim) list. value = n(n-1)/2 pairs per step x
steps x ranks / device time (inputs already in HBM). e2e is the same metric
through the C ABI with pinned host buffers: the CSR upload and the pair-list
download are inside the timed region.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --workload mixed_1m   # n = d = 1,000,000, Zipf(1.2), mean nnz 120
  python bench.py --workload batch      # 4,096 uneven instances, per-instance t
  python bench.py --workload serve      # 5M resident index, request server, p50/p99
Multi-GPU (torchrun): the default workload's self-join is split into row-block
shards (rank r takes the 128-row blocks b with b % N == r, cuapss_run_shard);
there is no cross-GPU exchange; value = the job's pairs / the slowest rank's
time (total work fixed: strong scaling). The batch and serve workloads run
one replica per rank.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "apss-cuda_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "APSS pairs/s (all-pairs throughput n(n-1)/2 / time, exact pair set vs FP64 oracle)"
WORKLOAD = "plain_800k"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), float(m["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampler run during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for ln in fh:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(x, t, p, budget_s=12.0):
    """OpenMP FP32 hybrid (oracle/oracle.c cpu_hybrid_apss) on a bounded
    sample of query rows of the same workload; extrapolated to the full job."""
    from oracle import oracle
    threads = oracle.max_threads()
    q = 32
    _, prep, qs = oracle.cpu_hybrid(x, t, p, 0, q, threads)
    per_row = max(qs / q, 1e-6)
    q = int(min(x.n, max(q, budget_s / per_row)))
    _, prep, qs = oracle.cpu_hybrid(x, t, p, 0, q, threads)
    covered = q * (x.n - 1) - q * (q - 1) / 2
    total = x.n * (x.n - 1) / 2
    full_time = prep + qs * total / covered
    return {"value": total / full_time, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": f"query rows 0..{q} of the workload against all j > i "
                      f"({covered:.3g} of {total:.3g} pairs, {qs:.1f} s) + full preprocessing "
                      f"({prep:.1f} s), extrapolated to the whole self-join"}


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU search (InvertedIndex_search,
    main.cu:104-141, built from its source into oracle/_ref/) on bounded
    samples of the workload, one process per host core group."""
    if rank != 0:
        return
    from cuapss import synth
    from oracle import oracle
    exe = oracle.ref_cpu_search_path()
    x = synth.generate(WORKLOAD, n=args.n) if args.n else synth.generate(WORKLOAD)
    total_pairs = x.n * (x.n - 1) / 2
    if exe is None:
        # no reference build here: time the CPU port instead
        vals = []
        for _ in range(args.warmup + args.steps):
            vals.append(cpu_baseline(x, args.t, 64, budget_s=8.0))
        v = vals[-args.steps:]
        value = sum(b["value"] for b in v) / len(v)
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "config": {"workload": WORKLOAD, "n": x.n, "t": args.t},
                "cpu_baseline": dict(v[-1], value=value),
                "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    nproc = max(1, min(os.cpu_count() or 1, 32))
    n_e = min(x.n, args.ref_index_rows)
    e = x.rows(0, n_e)
    td = tempfile.mkdtemp()
    pe = os.path.join(td, "e.csr")
    e.save(pe)

    def one_step(q_per_proc):
        procs, files = [], []
        for k in range(nproc):
            lo = n_e + k * q_per_proc
            if lo + q_per_proc > x.n:
                lo = (k * q_per_proc) % max(1, x.n - q_per_proc)
            b = x.rows(lo, lo + q_per_proc)
            pb = os.path.join(td, f"b{k}.csr")
            b.save(pb)
            files.append(pb)
            procs.append(subprocess.Popen([exe, pb, pe], stdout=subprocess.PIPE,
                                          stderr=subprocess.DEVNULL, text=True))
        secs = []
        for pr in procs:
            out, _ = pr.communicate()
            for ln in out.splitlines():
                if ln.startswith("search_seconds="):
                    secs.append(float(ln.split("=")[1]))
        if len(secs) != nproc:
            raise RuntimeError("reference harness failed")
        return max(secs)

    # calibrate: seconds per query row
    t1 = one_step(2)
    q = max(2, int(args.ref_step_s / max(t1 / 2, 1e-3)))
    for _ in range(args.warmup):
        one_step(q)
    times = [one_step(q) for _ in range(args.steps)]
    secs = sum(times) / len(times)
    ordered = nproc * q * n_e
    value = 0.5 * ordered / secs  # unordered-pair rate of a self-join by this method
    sample = (f"{nproc} processes x {q} query rows against the reference's inverted index of "
              f"{n_e} rows ({ordered:.3g} ordered pairs per step, {secs:.1f} s); a self-join "
              f"visits each unordered pair twice, so value = ordered rate / 2")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": x.n, "d": x.d, "t": 0.8,
                       "note": "the reference's CPU search has t = 0.8 hard-coded"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": nproc,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_batch(args, rank, world, local):
    """--workload batch: 4,096 independent instances (n log-uniform in
    [64, 20,000], d = 30,000, thresholds uniform in [0.6, 0.95]) in one
    cuapss_batch_run per step. value = sum of n_q(n_q-1)/2 per step / device
    time. Compared with launching the plain FP32 path once per instance."""
    import numpy as np
    import torch

    import cuapss
    from cuapss import synth

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    x, ip, tq = synth.generate_batch(k=args.k, seed=0)
    ns = np.diff(ip)
    pairs_per_step = float((ns * (ns - 1) // 2).sum())
    prec = cuapss.PREC_MIXED if args.precision == "mixed" else cuapss.PREC_FP32
    dev = {"rowptr": torch.from_numpy(x.rowptr).cuda(), "col": torch.from_numpy(x.col).cuda(),
           "val": torch.from_numpy(x.val).cuda(), "d": x.d}
    stream = torch.cuda.Stream()
    ctx = cuapss.Context(device=local, precision=prec, head_width=args.head,
                         stream=stream.cuda_stream)

    def alloc(c):
        return {"i": torch.empty(c, dtype=torch.int32, device="cuda"),
                "j": torch.empty(c, dtype=torch.int32, device="cuda"),
                "sim": torch.empty(c, dtype=torch.float32, device="cuda")}

    cap = 1 << 22
    out = alloc(cap)

    def step():
        nonlocal out, cap
        while True:
            try:
                return ctx.batch_run_device(dev, ip, tq, out)
            except cuapss.CuapssError as e:
                if e.status != cuapss.EOVERFLOW:
                    raise
                cap = ctx.required + 1024
                out = alloc(cap)

    for _ in range(max(args.warmup, 1)):  # the first call runs the autotuner
        npairs = step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            npairs = step()
            stats.append(dict(ctx.last_stats))
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        tms = torch.tensor([ms], device="cuda")
        dist.all_reduce(tms, op=dist.ReduceOp.MAX)
        ms = float(tms.item())
    value = world * pairs_per_step / (ms / 1e3)
    clocks = clk.summary()
    bucket_p = [int(v) for v in ctx.last_bucket_p]

    e2e = None
    if not args.no_e2e:
        hp = {"rowptr": torch.from_numpy(x.rowptr).pin_memory(),
              "col": torch.from_numpy(x.col).pin_memory(),
              "val": torch.from_numpy(x.val).pin_memory()}
        hcap = max(npairs, 1)
        ho = {"i": torch.empty(hcap, dtype=torch.int32).pin_memory(),
              "j": torch.empty(hcap, dtype=torch.int32).pin_memory(),
              "sim": torch.empty(hcap, dtype=torch.float32).pin_memory()}
        desc = cuapss.CsrDesc(x.n, x.d, x.nnz, hp["rowptr"].data_ptr(), hp["col"].data_ptr(),
                              hp["val"].data_ptr(), 0)
        ipc = np.ascontiguousarray(ip, np.int64)
        tqc = np.ascontiguousarray(tq, np.float32)
        L = cuapss.lib()

        def hstep():
            pr = cuapss.PairsDesc(ho["i"].data_ptr(), ho["j"].data_ptr(), ho["sim"].data_ptr(),
                                  hcap, 0, 0)
            s = L.cuapss_batch_run(ctx._h, ctypes.byref(desc), int(len(tqc)), ipc.ctypes.data,
                                   tqc.ctypes.data, ctypes.byref(pr), None, None)
            if s != cuapss.OK:
                raise cuapss.CuapssError(s, "cuapss_batch_run (host buffers)")
            return int(pr.count)

        hstep()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            hn = hstep()
        f1.record(stream)
        torch.cuda.synchronize()
        ems = f0.elapsed_time(f1) / args.steps
        if dist:
            tms = torch.tensor([ems], device="cuda")
            dist.all_reduce(tms, op=dist.ReduceOp.MAX)
            ems = float(tms.item())
        e2e = {"value": pairs_per_step / (ems / 1e3), "unit": "pairs/s",
               "ms_per_step": ems,
               "h2d_bytes_per_step": int(x.rowptr.nbytes + x.col.nbytes + x.val.nbytes +
                                         ipc.nbytes + tqc.nbytes),
               "d2h_bytes_per_step": int(hn * 12)}

    hbm, bf16, src = peaks()
    tile_ms = sum(s["ms_tiles"] for s in stats) / len(stats)
    s0 = stats[-1]
    tiles = int(s0["tiles"])
    if prec == cuapss.PREC_MIXED:
        # head GEMM flops of the tiles actually run: 2 * 128 * 128 * p per
        # tile, p of the bucket that owns the most tiles (stats.head_width)
        flops = 2.0 * 128 * 128 * int(s0["head_width"]) * tiles
        achieved = flops / (tile_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                    "frac": achieved / bf16, "traffic": None, "peak_source": src,
                    "kernel": "k_tiles_mma", "kernel_ms": tile_ms, "algorithmic_flops": flops,
                    "note": "tensor-core head flops of the 128x128 tiles over the tile-graph "
                            "time (one launch per size bucket)"}
    else:
        alg_bytes = 8.0 * s0["tail_products"] + 12.0 * s0["candidates"]
        achieved_gbs = alg_bytes / (tile_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                    "frac": achieved_gbs / hbm, "traffic": None, "peak_source": src,
                    "kernel": "k_tiles_fp32", "kernel_ms": tile_ms}

    # ---- comparison: the plain FP32 path launched once per instance
    per_inst = None
    if not args.no_plain:
        pctx = cuapss.Context(device=local, precision=cuapss.PREC_FP32, stream=stream.cuda_stream)
        insts = []
        for q in range(len(tq)):
            lo, hi = int(ip[q]), int(ip[q + 1])
            e_0, e_1 = int(x.rowptr[lo]), int(x.rowptr[hi])
            insts.append((q, {"rowptr": torch.from_numpy(x.rowptr[lo:hi + 1] - e_0).cuda(),
                              "col": dev["col"][e_0:e_1], "val": dev["val"][e_0:e_1],
                              "d": x.d}))
        pout = alloc(max(cap, 1 << 20))
        for q, d in insts[:16]:
            pctx.run_device(d, float(tq[q]), pout)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        tot = 0
        for q, d in insts:
            tot += pctx.run_device(d, float(tq[q]), pout)
        g1.record(stream)
        torch.cuda.synchronize()
        pms = g0.elapsed_time(g1)
        per_inst = {"value": world * pairs_per_step / (pms / 1e3), "unit": "pairs/s",
                    "ms_per_step": pms, "pairs_found": tot,
                    "same_pair_count_as_batch": tot == npairs,
                    "batch_over_per_instance": pms / ms,
                    "note": "cuapss_run (plain FP32) once per instance, inputs resident"}
        pctx.close()

    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == cuapss.PREC_FP32 else "bf16 head + f32 tail + f64 band",
        "data": "synthetic (seeded generator, independent row stream per instance)",
        "config": {"workload": "batch", "instances": int(len(tq)), "rows": x.n, "d": x.d,
                   "nnz": x.nnz, "n_range": [int(ns.min()), int(ns.max())],
                   "t_range": [float(tq.min()), float(tq.max())], "precision": args.precision,
                   "bucket_head_width": bucket_p,
                   "l2": "inputs larger than L2 (3.3 GB CSR)",
                   "parallelism": f"replicas x{world}"},
        "pairs_found": npairs, "candidates": s0["candidates"], "rescored": s0["rescored"],
        "tiles": tiles,
        "stage_ms": {k: sum(s[k] for s in stats) / len(stats)
                     for k in ("ms_preprocess", "ms_tiles", "ms_finalize", "ms_total")},
        "gpu_launches": int(sum(s["launches"] for s in stats)),
        "clocks": clocks, "roofline": roofline, "e2e": e2e, "per_instance_fp32": per_inst,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        threads = oracle.max_threads()
        rng = np.random.default_rng(7)
        done_pairs, secs, used = 0.0, 0.0, 0
        for q in rng.permutation(len(tq)):
            lo, hi = int(ip[q]), int(ip[q + 1])
            _, sp, sq = oracle.cpu_hybrid(x.rows(lo, hi), float(tq[q]), 128, 0, hi - lo, threads)
            secs += sp + sq
            done_pairs += (hi - lo) * (hi - lo - 1) / 2
            used += 1
            if secs > 12.0:
                break
        line["cpu_baseline"] = {"value": done_pairs / secs, "unit": "pairs/s", "cores": threads,
                                "kind": "port",
                                "sample": f"{used} random instances of the batch, each a full "
                                          f"self-join ({done_pairs:.3g} pairs, {secs:.1f} s)"}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


def run_serve(args, rank, world, local):
    """--workload serve: a resident index of 5,000,000 vectors (d = 2^20,
    nnz lognormal mean 60, Zipf 1.1) behind the request server. Requests
    arrive as a Poisson process; each is a query batch (log-uniform 1..4,096
    queries, per-query t uniform in [0.6, 0.95]) or, for 10% of them, an
    append of 1,000..50,000 vectors. Latency = submit -> results on the host
    (wall clock, the server's own record). value = query rows / wall time of
    the 256-query scenario at the highest offered load whose p99 stays within
    50 ms. Compared with the plain FP32 path answering each request alone."""
    import threading

    import numpy as np
    import torch

    import cuapss
    from cuapss import synth

    torch.cuda.set_device(local)
    if rank != 0:
        return
    n_index = args.n or 5_000_000
    cfg = synth.CONFIGS["serve_5m"]
    t0 = time.time()
    x = synth.generate(cfg, n=n_index)
    gen_s = time.time() - t0
    rng = np.random.default_rng(0)
    qoff = [50_000_000]

    def queries(m):
        q = synth.generate(cfg, n=m, row_offset=qoff[0])
        qoff[0] += m
        return q, rng.uniform(0.6, 0.95, size=m).astype(np.float32)

    aoff = [n_index]

    def append_rows(m):
        a = synth.generate(cfg, n=m, row_offset=aoff[0])
        aoff[0] += m
        return a

    def pct(v, p):
        return float(np.percentile(np.asarray(v), p)) if len(v) else None

    def drive(srv, reqs, rate):
        """Submit reqs (kind, csr, t) at Poisson times of the given rate
        (requests/s); returns per-request info and the wall time."""
        gaps = rng.exponential(1.0 / rate, size=len(reqs))
        infos = [None] * len(reqs)
        tickets = [None] * len(reqs)
        done = threading.Event()

        def collect():
            for k in range(len(reqs)):
                while tickets[k] is None:
                    time.sleep(0.0005)
                _, infos[k] = srv.wait(tickets[k], capacity=1 << 20)
            done.set()

        th = threading.Thread(target=collect)
        th.start()
        start = time.time()
        at = start
        for k, (kind, q, t) in enumerate(reqs):
            at += gaps[k]
            dt = at - time.time()
            if dt > 0:
                time.sleep(dt)
            tickets[k] = srv.submit_append(q) if kind == "append" else srv.submit_query(q, t)
        done.wait()
        th.join()
        return infos, time.time() - start

    def summarize(reqs, infos, wall):
        lat = [i["latency_ms"] for (k, _, _), i in zip(reqs, infos) if k == "query"]
        rows = sum(q.n for k, q, _ in reqs if k == "query")
        bat = [i["batch_rows"] for (k, _, _), i in zip(reqs, infos) if k == "query"]
        return {"requests": len(lat), "query_rows": rows, "queries_per_s": rows / wall,
                "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "max_ms": max(lat),
                "mean_batch_rows": float(np.mean(bat)), "wall_s": wall}

    out = {}
    with cuapss.Context(device=local, precision=cuapss.PREC_MIXED) as ctx:
        t1 = time.time()
        idx = cuapss.Index(ctx, x)
        torch.cuda.synchronize()
        build_s = time.time() - t1
        info0 = idx.info()
        # service time of a lone 256-query request (warm)
        q256, t256 = queries(256)
        for _ in range(3):
            idx.query(q256, t256)
        lone = []
        for _ in range(5):
            a = time.time()
            idx.query(q256, t256)
            lone.append((time.time() - a) * 1e3)
        lone_ms = float(np.median(lone))
        # scenario A: 256-query requests at offered loads relative to the
        # lone service rate (1.0 = one request in flight at a time)
        with cuapss.Server(idx, device=local, lanes=3) as srv:
            # warm-up: every lane's first batches grow its working memory
            warm = [srv.submit_query(*queries(1024)) for _ in range(9)]
            for tk in warm:
                srv.wait(tk, capacity=1 << 20)
            sweep = []
            with Clocks(local) as clk:
                for factor in (0.5, 1.0, 2.0, 4.0):
                    reqs = [("query",) + queries(256) for _ in range(args.serve_requests)]
                    rate = factor * 1000.0 / lone_ms
                    infos, wall = drive(srv, reqs, rate)
                    sweep.append(dict(summarize(reqs, infos, wall), offered_requests_per_s=rate,
                                      load_factor=factor))
            clocks = clk.summary()
            ok = [r for r in sweep if r["p99_ms"] <= 50.0]
            out["q256"] = max(ok, key=lambda r: r["queries_per_s"]) if ok else sweep[0]
            out["q256_sweep"] = sweep
            # scenario B: the mixed request stream with appends
            reqs = []
            for _ in range(args.serve_requests):
                if rng.uniform() < 0.1:
                    m = int(np.exp(rng.uniform(np.log(1000), np.log(50_000))))
                    reqs.append(("append", append_rows(m), None))
                else:
                    m = int(np.exp(rng.uniform(0, np.log(4096))))
                    reqs.append(("query",) + queries(max(1, m)))
            mean_rows = np.mean([q.n for k, q, _ in reqs if k == "query"])
            rate = 0.5 * (256.0 / lone_ms * 1000.0) / mean_rows
            infos, wall = drive(srv, reqs, rate)
            out["mix"] = dict(summarize(reqs, infos, wall), offered_requests_per_s=rate,
                              appends=sum(k == "append" for k, _, _ in reqs))
        info1 = idx.info()
        idx.close()
    # plain FP32 per-request path: each request alone, in arrival order
    plain = None
    if not args.no_plain:
        with cuapss.Context(device=local, precision=cuapss.PREC_FP32) as pctx:
            pidx = cuapss.Index(pctx, x)
            qs = [queries(256) for _ in range(max(5, args.serve_requests // 10))]
            pidx.query(*qs[0])
            lat = []
            for q, t in qs:
                a = time.time()
                pidx.query(q, t)
                lat.append((time.time() - a) * 1e3)
            plain = {"p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                     "queries_per_s": 256 * len(lat) / (sum(lat) / 1e3),
                     "note": "FP32 index, each 256-query request alone (service time)"}
            pidx.close()
    line = {
        "metric": "serving: queries/s at p99 <= 50 ms (256-query requests), 5M-vector "
                  "resident index; p50/p99 ms",
        "value": out["q256"]["queries_per_s"], "unit": "queries/s", "n_gpus": 1,
        "steps": args.serve_requests, "warmup": 3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 head + f32 tail + f64 band",
        "data": "synthetic (seeded generator; queries are fresh rows of the index's stream)",
        "config": {"workload": "serve", "index_rows": n_index, "d": x.d, "nnz": x.nnz,
                   "head_width": info0["head_width"], "lanes": 3,
                   "index_build_s": build_s, "generate_s": gen_s,
                   "index_device_bytes": info0["device_bytes"],
                   "segments_after": info1["segments"], "rows_after": info1["rows"]},
        "latency_ms": {"p50": out["q256"]["p50_ms"], "p99": out["q256"]["p99_ms"]},
        "lone_256_query_ms": lone_ms, "scenarios": out, "plain_fp32": plain, "clocks": clocks,
        "gpu_launches": None,
        "e2e": {"value": out["q256"]["queries_per_s"], "unit": "queries/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "requests are host CSR in, host pair lists out: every latency is "
                        "end to end"},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuapss", choices=["cuapss", "reference"])
    ap.add_argument("--t", type=float, default=0.7)
    ap.add_argument("--n", type=int, default=0, help="override n (smaller quick runs)")
    ap.add_argument("--head", type=int, default=0, help="head width p (0: library default)")
    ap.add_argument("--precision", default="mixed", choices=["fp32", "mixed"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ref-index-rows", type=int, default=100_000)
    ap.add_argument("--ref-step-s", type=float, default=8.0)
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=["plain_800k", "mixed_1m", "batch", "serve"],
                    help="plain_800k (default); mixed_1m: n = d = 1M; batch: 4,096 instances; "
                         "serve: 5M-vector resident index behind the request server")
    ap.add_argument("--serve-requests", type=int, default=400)
    ap.add_argument("--k", type=int, default=4096, help="instances of the batch workload")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batch" and args.impl == "cuapss":
        run_batch(args, rank, world, local)
        return
    if args.workload == "serve" and args.impl == "cuapss":
        run_serve(args, rank, world, local)
        return
    workload = args.workload if args.workload not in ("batch", "serve") else WORKLOAD
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch

    import cuapss
    from cuapss import synth

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    x = synth.generate(workload, n=args.n) if args.n else synth.generate(workload)
    prec = cuapss.PREC_MIXED if args.precision == "mixed" else cuapss.PREC_FP32
    dev = {"rowptr": torch.from_numpy(x.rowptr).cuda(), "col": torch.from_numpy(x.col).cuda(),
           "val": torch.from_numpy(x.val).cuda(), "d": x.d}
    stream = torch.cuda.Stream()
    ctx = cuapss.Context(device=local, precision=prec, head_width=args.head,
                         stream=stream.cuda_stream)
    cap = 1 << 22
    out = None

    def alloc(c):
        return {"i": torch.empty(c, dtype=torch.int32, device="cuda"),
                "j": torch.empty(c, dtype=torch.int32, device="cuda"),
                "sim": torch.empty(c, dtype=torch.float32, device="cuda")}

    out = alloc(cap)

    def step():
        nonlocal out, cap
        while True:
            try:
                if world > 1:  # this rank's shard of the one self-join
                    return ctx.run_shard_device(dev, args.t, rank, world, out)
                return ctx.run_device(dev, args.t, out)
            except cuapss.CuapssError as e:
                if e.status != cuapss.EOVERFLOW:
                    raise
                cap = ctx.required + 1024
                out = alloc(cap)

    for _ in range(max(args.warmup, 1)):
        npairs = step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            npairs = step()
            stats.append(dict(ctx.last_stats))
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        tms = torch.tensor([ms], device="cuda")
        dist.all_reduce(tms, op=dist.ReduceOp.MAX)
        ms = float(tms.item())
    # the job is one self-join of x; with N ranks each evaluates its shard
    pairs_per_step = x.n * (x.n - 1) / 2
    value = pairs_per_step / (ms / 1e3)
    clocks = clk.summary()

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        hp = {"rowptr": torch.from_numpy(x.rowptr).pin_memory(),
              "col": torch.from_numpy(x.col).pin_memory(),
              "val": torch.from_numpy(x.val).pin_memory()}
        hcap = max(npairs, 1)
        ho = {"i": torch.empty(hcap, dtype=torch.int32).pin_memory(),
              "j": torch.empty(hcap, dtype=torch.int32).pin_memory(),
              "sim": torch.empty(hcap, dtype=torch.float32).pin_memory()}
        desc = cuapss.CsrDesc(x.n, x.d, x.nnz, hp["rowptr"].data_ptr(), hp["col"].data_ptr(),
                              hp["val"].data_ptr(), 0)
        L = cuapss.lib()

        def hstep():
            pr = cuapss.PairsDesc(ho["i"].data_ptr(), ho["j"].data_ptr(), ho["sim"].data_ptr(),
                                  hcap, 0, 0)
            if world > 1:
                s = L.cuapss_run_shard(ctx._h, ctypes.byref(desc), ctypes.c_float(args.t), rank,
                                       world, ctypes.byref(pr), None)
            else:
                s = L.cuapss_run(ctx._h, ctypes.byref(desc), ctypes.c_float(args.t),
                                 ctypes.byref(pr), None)
            if s != cuapss.OK:
                raise cuapss.CuapssError(s, "cuapss_run (host buffers)")
            return int(pr.count)

        hstep()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            hn = hstep()
        f1.record(stream)
        torch.cuda.synchronize()
        ems = f0.elapsed_time(f1) / args.steps
        if dist:
            tms = torch.tensor([ems], device="cuda")
            dist.all_reduce(tms, op=dist.ReduceOp.MAX)
            ems = float(tms.item())
        e2e = {"value": world * pairs_per_step / (ems / 1e3), "unit": "pairs/s",
               "ms_per_step": ems,
               "h2d_bytes_per_step": int(x.rowptr.nbytes + x.col.nbytes + x.val.nbytes),
               "d2h_bytes_per_step": int(hn * 12)}

    # ---- roofline of the dominant kernel (the pair-tile kernel) ----
    hbm, bf16, src = peaks()
    tile_ms = sum(s["ms_tiles"] for s in stats) / len(stats)
    s0 = stats[-1]
    p = int(s0["head_width"])
    head_flops = 2.0 * p * pairs_per_step  # BF16/FP32 multiply-adds of the head dot
    if world > 1:  # this rank's share: its tiles of the triangle's tiles
        nb = (x.n + 127) // 128
        head_flops *= s0["tiles"] / (nb * (nb + 1) / 2)
    if prec == cuapss.PREC_MIXED:
        achieved = head_flops / (tile_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                    "frac": achieved / bf16, "traffic": None, "peak_source": src,
                    "kernel": "k_tiles_mma", "kernel_ms": tile_ms,
                    "algorithmic_flops": head_flops,
                    "note": "head BF16 GEMM flops 2*p*n(n-1)/2 over the tile-kernel time "
                            "(the kernel also runs the sparse FP32 tail and the epilogue)"}
    else:
        alg_bytes = 8.0 * s0["tail_products"] + 4.0 * p * x.n + 12.0 * s0["candidates"]
        achieved_gbs = alg_bytes / (tile_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                    "frac": achieved_gbs / hbm, "traffic": None, "peak_source": src,
                    "kernel": "k_tiles_fp32", "kernel_ms": tile_ms,
                    "algorithmic_bytes": alg_bytes,
                    "note": "FP32 head runs on CUDA cores (FMA-bound); head FP32 FMA rate "
                            f"{head_flops / (tile_ms / 1e3) / 1e12:.1f} TFLOP/s"}

    # ---- the plain FP32 hybrid on the same data (the mixed path's comparison)
    plain = None
    if prec == cuapss.PREC_MIXED and not args.no_plain and world == 1:
        pctx = cuapss.Context(device=local, precision=cuapss.PREC_FP32, stream=stream.cuda_stream)
        pout = alloc(cap)
        pctx.run_device(dev, args.t, pout)
        pstats = []
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(max(1, args.steps // 2)):
            pn = pctx.run_device(dev, args.t, pout)
            pstats.append(dict(pctx.last_stats))
        g1.record(stream)
        torch.cuda.synchronize()
        pms = g0.elapsed_time(g1) / max(1, args.steps // 2)
        same = bool(pn == npairs and torch.equal(pout["i"][:pn], out["i"][:npairs]) and
                    torch.equal(pout["j"][:pn], out["j"][:npairs]))
        plain = {"value": pairs_per_step / (pms / 1e3), "unit": "pairs/s",
                 "ms_per_step": pms, "head_width": int(pstats[-1]["head_width"]),
                 "pairs_found": pn, "same_pair_set_as_mixed": same,
                 "mixed_over_plain": pms / ms}
        pctx.close()

    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if prec == cuapss.PREC_FP32 else "bf16 head + f32 tail + f64 band",
        "data": "synthetic (seeded generator, reference corpus not distributed)",
        "config": {"workload": workload, "n": x.n, "d": x.d, "nnz": x.nnz, "t": args.t,
                   "precision": args.precision, "head_width": p,
                   "l2": "inputs larger than L2 (CSR + head block > 126 MB)",
                   "parallelism": f"row-block shards x{world}" if world > 1 else "1 GPU"},
        "pairs_found": npairs, "candidates": s0["candidates"], "rescored": s0["rescored"],
        "stage_ms": {k: sum(s[k] for s in stats) / len(stats)
                     for k in ("ms_preprocess", "ms_tiles", "ms_finalize", "ms_total")},
        "gpu_launches": int(sum(s["launches"] for s in stats)),
        "clocks": clocks, "roofline": roofline, "e2e": e2e, "plain_fp32": plain,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(x, args.t, 128)  # the CPU's own best head width
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
