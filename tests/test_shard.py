"""Sharding of the self-join across processes (one per GPU): the host-side
block partition, checked by two gloo ranks on CPU, and the GPU shards'
outputs, which are disjoint and add up to the single-process result."""
import datetime
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import cuapss
from cuapss import synth


def _rank_blocks(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mine = [int(b) for b in cuapss.shard_blocks(n, rank, world)]
    objs = [None] * world
    dist.all_gather_object(objs, mine)
    if rank == 0:
        q.put(objs)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("n", [1, 129, 100_000])
def test_two_gloo_ranks_partition_blocks(n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (n % 1000)
    procs = [ctx.Process(target=_rank_blocks, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    objs = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    nb = (n + 127) // 128
    allb = sorted(objs[0] + objs[1])
    assert allb == list(range(nb))  # disjoint and complete
    assert abs(len(objs[0]) - len(objs[1])) <= 1
    # the triangle's tiles split evenly: rank 0 holds at most one row more
    tiles = [sum(nb - b for b in o) for o in objs]
    assert abs(tiles[0] - tiles[1]) <= nb


def test_shard_blocks_arguments():
    assert cuapss.shard_blocks(0, 0, 1).size == 0
    with pytest.raises(ValueError):
        cuapss.shard_blocks(10, 2, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [cuapss.PREC_MIXED, cuapss.PREC_FP32], ids=["mixed", "fp32"])
def test_shards_union_is_the_full_join(precision):
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    x = synth.generate("plain_20k", n=3000, dup_frac=0.2)
    with cuapss.Context(precision=precision) as c:
        full = c.run(x, 0.6)
        for nshards in (1, 2, 3, 8):
            parts = [c.run_shard(x, 0.6, s, nshards) for s in range(nshards)]
            for s, (i, j, _) in enumerate(parts):
                assert np.all((i // 128) % nshards == s)
            key = np.concatenate([p[0].astype(np.int64) * x.n + p[1] for p in parts])
            order = np.argsort(key)
            assert np.array_equal(key[order], full[0].astype(np.int64) * x.n + full[1])
            sims = np.concatenate([p[2] for p in parts])[order]
            assert np.array_equal(sims, full[2])
