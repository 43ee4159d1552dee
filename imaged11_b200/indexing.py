"""Trial-orientation scoring for an ImageD11 indexer, batched.

``indexer.scorethem`` (ImageD11/indexing.py:762-874) walks its list of hits
(pairs of peaks i, j on two rings) one at a time: orient a cell on the pair,
score the orientation against every g-vector, and -- for those above minpks --
re-orient over the angle window, refine, and keep the grain when enough of its
peaks are new.  The score of the first orientation of every hit depends on
nothing the loop changes, so ``scorethem`` below computes all of them first
and scores them in one GPU launch (the cell index, or the FP32 screening
kernel); the walk that follows makes the reference's decisions in the
reference's order with those counts, calling the indexer's own methods for
everything else.  The result -- ubis, scores and peak assignments ga -- is the
one the reference's loop produces.

``idx`` is an ImageD11 ``indexing.indexer`` or any object with its attributes
(hits, ga, gv, gvflat, hkl_tol, minpks, max_grains, uniqueness, ubis, scores,
ring_1, ring_2, cosine_tol, unitcell with orient/UBI/UBIlist) and methods
(score, getind).
"""
import numpy as np

from . import batch, cImageD11


def trial_orientations(idx, hits):
    """UBI of the first orientation (unitcell.orient without an angle window)
    for each hit (diff, i, j); None where i == j (the reference skips those)."""
    out = []
    for _, i, j in hits:
        if i == j:
            out.append(None)
            continue
        idx.unitcell.orient(idx.ring_1, idx.gv[i, :], idx.ring_2, idx.gv[j, :], verbose=0)
        out.append(np.array(idx.unitcell.UBI, dtype=np.float64).copy())
    return out


def scorethem(idx, method="grid"):
    """Drop-in for indexer.scorethem (without the fitb4 option); returns the
    number of grains kept.  method: "grid" (cell index) or "screen" (FP32
    screening kernel) for the batched first-pass scores."""
    if idx.hits is None or len(idx.hits) == 0:
        return 0
    tol = float(idx.hkl_tol)
    order = list(reversed(idx.hits))        # the reference pops from the end
    ubis = trial_orientations(idx, order)
    valid = [k for k, u in enumerate(ubis) if u is not None]
    npk_first = np.zeros(len(order), np.int64)
    if valid:
        stack = np.stack([ubis[k] for k in valid])
        if method == "grid":
            counts = batch.score_grid(stack, batch.GvecGrid(idx.gv), [tol])
        else:
            counts = batch.score_batch(stack, batch.GvecSet(idx.gv), [tol])
        npk_first[valid] = counts[:, 0].cpu().numpy()
    gv = idx.gvflat
    drlv2tmp = np.empty(len(idx.gv), float)
    labelstmp = np.empty(len(idx.gv), np.int32)
    kept = 0
    k_end = len(order)
    for k, (_, i, j) in enumerate(order):
        if kept >= idx.max_grains:
            k_end = k
            break
        if idx.ga[i] > -1 or idx.ga[j] > -1 or i == j:
            continue
        ubi = ubis[k]
        npk = int(npk_first[k])
        if npk <= idx.minpks:
            continue
        # orientations within the angle window; the best of them if it scores
        # at least as well as the first
        idx.unitcell.orient(idx.ring_1, idx.gv[i, :], idx.ring_2, idx.gv[j, :], verbose=0,
                            crange=abs(idx.cosine_tol))
        if len(idx.unitcell.UBIlist) > 1:
            npks = [idx.score(u, tol) for u in idx.unitcell.UBIlist]
            c = int(np.argmax(npks))
            if npks[c] >= npk:
                ubi = np.array(idx.unitcell.UBIlist[c], dtype=np.float64).copy()
                npk = npks[c]
        ubi = np.ascontiguousarray(ubi, dtype=np.float64)
        cImageD11.score_and_refine(ubi, gv, tol)
        ind = idx.getind(ubi, drlv2tmp=drlv2tmp, labelstmp=labelstmp)
        ga = idx.ga[ind]
        uniqueness = np.sum(np.where(ga == -1, 1, 0)) * 1.0 / ga.shape[0]
        if uniqueness > idx.uniqueness:
            idx.ga[ind] = len(idx.scores) + 1
            idx.ubis.append(ubi)
            idx.scores.append(npk)
            kept += 1
    idx.hits = list(reversed(order[k_end:]))  # what the reference leaves unpopped
    if len(idx.ubis) > 0 and hasattr(idx, "refine"):
        idx.refine(idx.ubis[int(np.argmax(idx.scores))])  # as the reference ends
    return kept
