"""Multi-GPU sharding of batched scoring over trial UBIs (one process per GPU).

Trial UBIs are independent, so the scoring work shards by UBI with the
g-vectors replicated on every rank and no exchange on the data path.  This
module holds the host-side logic: contiguous shard ranges and the all-gather
of per-rank counts when every rank needs the full table (an indexing driver
deciding which trials to keep).  The per-rank scorer is passed in, normally
``lambda u: batch.score_batch(u, gvec_set, tols)``.
"""
import numpy as np


def shard_range(m, rank, world):
    """[lo, hi) of the rank's contiguous share of m items (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world %d/%d" % (rank, world))
    base, extra = divmod(m, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def score_sharded(ubis, ntol, scorer, group=None, device=None):
    """Score this rank's share of ``ubis`` with ``scorer`` and all-gather the
    counts so every rank returns the full (m, ntol) int32 table (numpy).

    ``device``: where the collective's buffers live ("cuda" for NCCL, "cpu"
    for gloo); defaults from the process group's backend."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    m = len(ubis)
    lo, hi = shard_range(m, rank, world)
    local = np.asarray(scorer(ubis[lo:hi]), dtype=np.int32).reshape(hi - lo, ntol)
    width = -(-m // world)                      # largest shard
    buf = torch.zeros((width, ntol), dtype=torch.int32, device=device)
    buf[: hi - lo] = torch.as_tensor(local, device=device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty((m, ntol), np.int32)
    for r, p in enumerate(parts):
        a, b = shard_range(m, r, world)
        out[a:b] = p[: b - a].cpu().numpy()
    return out
