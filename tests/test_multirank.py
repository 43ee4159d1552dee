"""Multi-rank (world_size 2 and 3) sharding of batched scoring over UBIs, on
CPU with the gloo backend.  The per-rank scorer is the oracle here; on GPUs it
is the CUDA batch scorer -- the sharding and gather logic is the same."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from imaged11_b200 import shard
        from oracle.oracle import Oracle
        d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "scoring.npz")))
        orc = Oracle()
        tols = d["sc_tols"][:3]
        got = shard.score_sharded(d["sc_ubis"], len(tols),
                                  lambda u: orc.score_many(u, d["sc_gv"], tols))
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_score_sharded_gloo(world, golden):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = golden["scoring"]["sc_counts"][:, :3]
    for r in range(world):
        assert np.array_equal(results[r], want)


def test_shard_range_partitions():
    from imaged11_b200 import shard
    for m in (0, 1, 7, 20000, 20001):
        for world in (1, 2, 3, 8):
            spans = [shard.shard_range(m, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == m
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
