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


class NumpyAssignPasses:
    """The per-rank assignment passes restated in numpy (the reference's FP64
    operation order for drlv2), for the CPU test of the exchange logic."""

    def __init__(self, gv):
        self.gv = np.ascontiguousarray(gv, dtype=np.float64)

    def _drlv2(self, u):
        g = self.gv
        s = 0.0
        for r in range(3):
            h = u[r, 0] * g[:, 0] + u[r, 1] * g[:, 1] + u[r, 2] * g[:, 2]
            t = h - np.rint(h)
            s = s + t * t if r else t * t
        return s

    def run_pass(self, p, ubis_shard, base, tol, drlv2, best, lab):
        from imaged11_b200 import shard
        if p == -1:
            best.fill_(shard.NO_BEST)
            lab.fill_(shard.NO_LABEL)
            return
        d = drlv2.numpy()
        b = best.numpy()
        lb = lab.numpy()
        for i, u in enumerate(ubis_shard):
            s = self._drlv2(u)
            ok = (s < tol * tol) & (s < d)
            bits = s.view(np.int64)
            if p == 0:
                np.minimum(b, np.where(ok, bits, shard.NO_BEST), out=b)
            else:
                np.minimum(lb, np.where(ok & (bits == b), base + i, shard.NO_LABEL).astype(np.int32),
                           out=lb)

    def final(self, ubis_all, grain_labels, tol, best, lab, drlv2, labels, npk):
        from imaged11_b200 import shard
        gl = np.arange(len(ubis_all)) if grain_labels is None else np.asarray(grain_labels)
        lb, b = lab.numpy(), best.numpy()
        d, out = drlv2.numpy(), labels.numpy()
        won = lb != shard.NO_LABEL
        out[won] = gl[lb[won]]
        d[won] = b[won].view(np.float64)
        out[~won & np.isin(out, gl)] = -1


def _assign_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from imaged11_b200 import shard
        d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "scoring.npz")))
        n = len(d["sc_gv"])
        rng = np.random.default_rng(9)
        drlv2 = torch.tensor(rng.uniform(0.0, 0.03, n))
        labels = torch.tensor(rng.choice([-1, 3, 105, 115], n).astype(np.int32))
        gl = np.arange(len(d["sc_ubis"])) * 10 + 5
        shard.score_and_assign_sharded(d["sc_ubis"], 0.05, drlv2, labels,
                                       NumpyAssignPasses(d["sc_gv"]), grain_labels=gl)
        q.put((rank, drlv2.numpy().copy(), labels.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_assign_sharded_gloo(world, oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_assign_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, dd, ll = q.get(timeout=120)
        results[r] = (dd, ll)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "scoring.npz")))
    n = len(d["sc_gv"])
    rng = np.random.default_rng(9)
    ref_d = rng.uniform(0.0, 0.03, n)
    ref_l = rng.choice([-1, 3, 105, 115], n).astype(np.int32)
    for i, u in enumerate(d["sc_ubis"]):
        _, ref_d, ref_l = oracle.score_and_assign(u, d["sc_gv"], 0.05, ref_d, ref_l, i * 10 + 5)
    for r in range(world):
        assert np.array_equal(results[r][1], ref_l)
        assert np.array_equal(results[r][0], ref_d)
