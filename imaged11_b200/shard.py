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


# ---------------------------------------------------------------- assignment --
# Batched score_and_assign with the grains sharded over ranks.  Unlike scoring,
# assignment has a real exchange: every g goes to the first grain, over all
# ranks' grains, with the smallest drlv2.  Two MIN all-reduces over the
# g-vectors carry it -- of the best drlv2 (its FP64 bits, which order like the
# values for non-negative numbers, as int64) and then of the lowest global
# grain index reaching that best -- so every rank ends with the labels and
# drlv2 of the reference's sequence of calls over all grains.

NO_BEST = 0x7FFFFFFFFFFFFFFF
NO_LABEL = 2 ** 31 - 1


class CudaAssignPasses:
    """The per-rank passes on this rank's GPU through the cell index."""

    def __init__(self, grid):
        self.grid = grid

    def run_pass(self, p, ubis_shard, base, tol, drlv2, best, lab):
        from . import batch
        from ._lib import lib, check
        torch = batch._torch()
        u = batch._dev(ubis_shard, torch.float64).reshape(-1, 9)
        g = self.grid
        check(lib.id11b_dev_assign_grid_pass(u.data_ptr(), u.shape[0], int(base), g.n, g.nx,
                                             g.xsub, g.buf.data_ptr(), float(tol),
                                             drlv2.data_ptr(), int(p), best.data_ptr(),
                                             lab.data_ptr(), batch._stream()), "assign_pass")

    def final(self, ubis_all, grain_labels, tol, best, lab, drlv2, labels, npk):
        from . import batch
        from ._lib import lib, check
        torch = batch._torch()
        u = batch._dev(ubis_all, torch.float64).reshape(-1, 9)
        g = self.grid
        check(lib.id11b_dev_assign_grid_final(u.data_ptr(), u.shape[0],
                                              grain_labels.data_ptr() if grain_labels is not None
                                              else None, g.gv.data_ptr(), g.n, g.nx, g.xsub,
                                              g.buf.data_ptr(), float(tol), best.data_ptr(),
                                              lab.data_ptr(), drlv2.data_ptr(),
                                              labels.data_ptr(),
                                              npk.data_ptr() if npk is not None else None,
                                              batch._stream()), "assign_final")


def score_and_assign_sharded(ubis, tol, drlv2, labels, passes, grain_labels=None, npk=None,
                             group=None, device=None):
    """drlv2 (n float64) and labels (n int32) updated in place, on every rank,
    to the result of score_and_assign (ImageD11 src/closest.c:366-397) called
    for grain i = 0 .. m-1 in order with label grain_labels[i] (default i).
    Every rank holds all m UBIs and the same inputs and works on its
    contiguous share of the grains; ``passes`` runs the per-rank work
    (CudaAssignPasses(grid) on a GPU).  ``device`` holds the collective's
    buffers ("cuda" for NCCL, "cpu" for gloo; from the backend by default)."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    m = len(ubis)
    n = drlv2.shape[0]
    lo, hi = shard_range(m, rank, world)
    work = drlv2.device
    best = torch.empty(n, dtype=torch.int64, device=work)
    lab = torch.empty(n, dtype=torch.int32, device=work)

    def reduce_min(t):
        buf = t.to(device)
        dist.all_reduce(buf, op=dist.ReduceOp.MIN, group=group)
        t.copy_(buf.to(work))

    passes.run_pass(-1, ubis[lo:hi], lo, tol, drlv2, best, lab)
    passes.run_pass(0, ubis[lo:hi], lo, tol, drlv2, best, lab)
    reduce_min(best)
    passes.run_pass(1, ubis[lo:hi], lo, tol, drlv2, best, lab)
    reduce_min(lab)
    passes.final(ubis, grain_labels, tol, best, lab, drlv2, labels, npk)
    return drlv2, labels
