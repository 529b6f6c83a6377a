"""Generate the golden fixtures that pin the CPU oracle to the reference.

The reference (fengyilin118/APSS-CUDA) ships no tests, no golden vectors and
no dataset. Its one CPU search, InvertedIndex_search (main.cu:104-141), is
compiled from the reference's own source by oracle/Makefile into
oracle/_ref/ref_cpu_search. This script runs it on seeded synthetic inputs
(partition B = query rows, partition E = indexed rows; its threshold is the
hard-coded 0.8) and records the pair count it prints, together with a digest
of the input so that a change of the generator is detected.

The GPU harness of the reference's index kernels (oracle/_ref/ref_index) is
run by the GPU test suite, not here (this container has no GPU).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "apss-cuda_b200"))
sys.path.insert(0, ROOT)

from cuapss import synth  # noqa: E402
from oracle import oracle  # noqa: E402

# (name, generator config, overrides, B rows, E rows)
CASES = [
    ("plain_20k_b0-3000_e3000-9000", "plain_20k", {}, (0, 3000), (3000, 9000)),
    ("plain_20k_b9000-12000_e0-9000", "plain_20k", {}, (9000, 12000), (0, 9000)),
    ("batch_instance_s7", "batch_instance", {"n": 6000, "seed": 7}, (3000, 6000), (0, 3000)),
    ("plain_800k_head_rows", "plain_800k", {"n": 8000, "nnz_max": 400}, (4000, 8000), (0, 4000)),
]


def digest(x) -> str:
    h = hashlib.sha256()
    for a in (x.rowptr, x.col, x.val):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run_reference(b, e) -> int:
    exe = oracle.ref_cpu_search_path()
    if exe is None:
        raise SystemExit("oracle/_ref/ref_cpu_search is not built (make -C oracle)")
    with tempfile.TemporaryDirectory() as td:
        pb, pe = os.path.join(td, "b.csr"), os.path.join(td, "e.csr")
        b.save(pb)
        e.save(pe)
        out = subprocess.run([exe, pb, pe], check=True, capture_output=True, text=True).stdout
    last = [ln for ln in out.splitlines() if ln.startswith("sum_pair=")]
    return int(last[-1].split("=")[1])


def main() -> None:
    cases = []
    for name, cfg, over, (b0, b1), (e0, e1) in CASES:
        x = synth.generate(cfg, **over)
        b, e = x.rows(b0, b1), x.rows(e0, e1)
        ref = run_reference(b, e)
        oi, oj, os_ = oracle.join(b, e, 0.0)
        near = float(np.min(np.abs(os_ - 0.8))) if len(os_) else 1.0
        cases.append({
            "name": name, "config": cfg, "overrides": over,
            "b_rows": [b0, b1], "e_rows": [e0, e1], "t": 0.8,
            "ref_sum_pair": ref,
            "closest_sim_to_t": near,
            "input_sha256": digest(x),
        })
        print(name, "reference sum_pair =", ref, "closest |sim-0.8| =", near)
    out = {
        "source": "oracle/_ref/ref_cpu_search = reference main.cu InvertedIndex_search "
                  "(main.cu:104-141), compiled from the reference tree",
        "cases": cases,
    }
    with open(os.path.join(ROOT, "tests", "golden", "ref_cpu_search.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
