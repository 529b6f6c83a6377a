"""bench.py's host-side plumbing on CPU: the multi-rank launcher (gloo, no
GPU) and the reference arm, which must map no library of the package."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out: str) -> dict:
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert lines, out
    return json.loads(lines[-1])


@pytest.mark.parametrize("gpus,n", [(2, 100_000), (3, 1_000)])
def test_launcher_starts_ranks_and_shards_partition_blocks(gpus, n):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", str(gpus),
                        "--dry-shards", "--n", str(n)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    line = _last_json(r.stdout)
    assert line["n_gpus"] == gpus
    assert line["partition_ok"]
    nb = (n + 127) // 128
    assert sum(line["shard_blocks"]) == nb
    assert sum(line["shard_tiles"]) == nb * (nb + 1) // 2
    assert max(line["shard_tiles"]) - min(line["shard_tiles"]) <= nb


def test_reference_arm_maps_only_oracle_libraries():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--n", "3000", "--steps", "1", "--warmup", "0", "--ref-step-s", "0.05"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = _last_json(r.stdout)
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["workload"] == "mixed_1m" and line["config"]["t"] == 0.7
    libs = line["mapped_repo_libraries"]
    assert libs and all(p.startswith("oracle" + os.sep) for p in libs), libs
    assert line["e2e"]["h2d_bytes_per_step"] == 0
