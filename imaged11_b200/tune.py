"""Autotuner for the launch shapes of the batched kernels.

The reference has no counterpart: it scores one UBI per call
(ImageD11 src/closest.c:227-248) and refines one grain per call
(src/closest.c:267-345).  Two shapes are tuned here, each by timing the
candidates with CUDA events on the caller's own inputs:

* score_batch tile -- UBIs per thread (2 or 4: 512 or 1,024 UBIs per CTA, held
  in registers) x gsplit (how many g ranges each block of UBIs is split
  into, i.e. how many 1,024-vector shared-memory tiles a CTA streams).
  Counts are identical for every tile shape, so tuning needs no reference.
* GrainSet CTA size for the persistent per-grain refinement (32..256).
* the cell index's shape (y/z cell side relative to about one g per cell, and
  how many times finer x is cut), timed with score_grid.

Results are cached per (device, shape bucket): m and n rounded up to powers of
two.  ``save``/``load`` persist the cache as JSON; setting
IMAGED11_B200_TUNE_CACHE to a file name loads it at import and makes
``tune_score``/``tune_refine`` write it back.
"""
import json
import math
import os

from ._lib import lib, check

_cache = {}
CACHE_ENV = "IMAGED11_B200_TUNE_CACHE"


def _torch():
    import torch
    return torch


def _bucket(x):
    return 1 << max(0, int(math.ceil(math.log2(max(int(x), 1)))))


def _device_name():
    torch = _torch()
    return torch.cuda.get_device_name(torch.cuda.current_device())


def score_key(m, n, ntol):
    return "score|%s|%d|%d|%d" % (_device_name(), _bucket(m), _bucket(n), int(ntol))


def refine_key(ngrains, peaks):
    return "refine|%s|%d|%d" % (_device_name(), _bucket(ngrains), _bucket(peaks))


def default_score_tile(m, n):
    """(UBIs per thread, gsplit) the built-in heuristic picks."""
    import ctypes
    r = ctypes.c_int(0)
    g = ctypes.c_int(0)
    check(lib.id11b_score_tile_default(int(m), int(n), ctypes.addressof(r), ctypes.addressof(g)),
          "score_tile_default")
    return r.value, g.value


def score_candidates(m, n):
    """Tile shapes tried by tune_score: both register blockings, each with the
    heuristic's g split scaled by 1/8 .. 4 (at most one tile per CTA)."""
    maxgs = max(1, -(-int(n) // 1024))
    out = []
    for r in (4, 2):
        per = 256 * r
        ublocks = max(1, -(-int(m) // per))
        # the heuristic's split for this blocking: ~16 waves of resident CTAs
        torch = _torch()
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        base = max(1, -(-(sms * (3 if r == 4 else 4) * 16) // ublocks))
        for f in (0.125, 0.25, 0.5, 1.0, 2.0, 4.0):
            gs = int(min(maxgs, max(1, round(base * f))))
            if (r, gs) not in out:
                out.append((r, gs))
    return out


def _time(fn, reps):
    torch = _torch()
    st = torch.cuda.current_stream()
    fn()  # warm-up (also loads the kernel)
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune_score(ubis, gvs, tols, reps=3, candidates=None):
    """Time every candidate tile shape of score_batch on these inputs, cache
    the fastest for this shape bucket and return (tile, [(tile, ms), ...])."""
    from . import batch
    torch = _torch()
    u = batch._dev(ubis, torch.float64).reshape(-1, 9)
    m = u.shape[0]
    ws = batch.BatchWorkspace(m, gvs.n, False)
    out = torch.empty((m, len(batch._tols(tols))), dtype=torch.int32, device=u.device)
    table = []
    for tile in candidates or score_candidates(m, gvs.n):
        ms = _time(lambda: batch.score_batch(u, gvs, tols, workspace=ws, out=out, tile=tile),
                   reps)
        table.append((tuple(tile), ms))
    best = min(table, key=lambda x: x[1])[0]
    _cache[score_key(m, gvs.n, len(batch._tols(tols)))] = list(best)
    _autosave()
    return best, table


def score_tile(m, n, ntol):
    """The tuned tile for this shape bucket, or None (use the heuristic)."""
    if not _cache:
        return None
    t = _cache.get(score_key(m, n, ntol))
    return tuple(t) if t else None


def tune_refine(grains, tol, iters, reps=3, threads=(32, 64, 128, 256)):
    """Time the persistent refinement of a GrainSet at each CTA size (UBIs are
    restored after every trial), set grains.threads to the fastest, cache it
    and return (threads, [(threads, ms), ...])."""
    saved = grains.ubis.clone()
    table = []
    for t in threads:
        def run():
            grains.ubis.copy_(saved)
            grains._launch(tol, iters, 1, t)
        table.append((t, _time(run, reps)))
    grains.ubis.copy_(saved)
    best = min(table, key=lambda x: x[1])[0]
    grains.threads = best
    _cache[refine_key(grains.ngrains, grains.peaks)] = best
    _autosave()
    return best, table


def refine_threads(ngrains, peaks):
    """The tuned CTA size for this shape bucket, or None."""
    if not _cache:
        return None
    return _cache.get(refine_key(ngrains, peaks))


def grid_key(n):
    return "grid|%s|%d" % (_device_name(), _bucket(n))


def halo_cell_factor(ubis, base, tmax):
    """The smallest y/z cell side, as a factor of base.cs, at which the binned
    join's halo is one row of cells each way: the join stages for each row of
    cells the g within W + 2 eps of it (W the largest widened box half width,
    eps = 2e-5 (1 + G)), over ceil((W + 2 eps) / cs) rows each way, and a
    second ring of rows multiplies the staging (measured: 20,000 UBIs x 1.1M g
    took 2.78 ms just above this side and 3.16 ms just below it).  W is
    estimated here as the enumeration widens each box: (tmax + 1e-6) times the
    norm of UB's row plus the FP32 centre margin 4 2^-24 max|hkl| sum|UB row|,
    over the UBIs the join takes (finite, invertible, with fewer candidate hkl
    than g).  None if no UBI qualifies."""
    torch = _torch()
    u = ubis.reshape(-1, 3, 3)
    if u.shape[0] == 0:
        return None
    det = torch.nan_to_num(torch.linalg.det(u).abs(), nan=0.0, posinf=0.0)
    ok = det > 0
    ub = torch.linalg.inv(torch.where(ok[:, None, None], u,
                                      torch.eye(3, dtype=u.dtype, device=u.device)))
    G = base.gmax * (1 + 1e-6)
    hm = (u.abs().sum(dim=2) * G + 1.0).ceil()                     # |hkl| bound per row
    ok &= (2 * hm + 1).prod(dim=1) <= base.n
    w = (tmax + 1e-6) * ub.norm(dim=2) * (1 + 1e-9) + \
        4 * 2.0 ** -24 * hm.max(dim=1, keepdim=True).values * ub.abs().sum(dim=2)
    w = torch.nan_to_num(w, nan=0.0, posinf=0.0).max(dim=1).values
    if not bool(ok.any()):
        return None
    W = float(torch.where(ok, w, torch.zeros_like(w)).max().item())
    eps = 2e-5 * (1 + G)
    return (W + 2 * eps) * (1 + 1e-3) / base.cs


def tune_grid(ubis, gv, tols, cell_factors=None, xsubs=(1, 2, 4, 8), reps=2, method=None):
    """Time score_grid on these inputs for cell-index shapes: y/z cell side =
    factor x the default (about one g per cell of the bounding cube) and x cut
    xsub times finer, and for its two methods; cache the fastest shape and
    method per g-count bucket (GvecGrid uses the shape when built without an
    explicit one, score_grid the method when called without one) and return
    ((factor, xsub), table of ((factor, xsub, method), ms)).  cell_factors:
    None tries 0.8, 1.0 and 1.25 and 1.0, 1.12, 1.25 and 1.5 times
    halo_cell_factor (the binned join's best sides lie just above it: 0.9 x the
    default for 20,000 UBIs x 1.1M g, 2 x for 10,000 x 10M).  method: time only
    that score_grid method ("bins" or "walk"; None: both, "bins" where the
    tolerances and the shape allow it)."""
    from . import batch
    torch = _torch()
    g = batch._dev(gv, torch.float64).reshape(-1, 3)
    u = batch._dev(ubis, torch.float64).reshape(-1, 9)
    base = batch.GvecGrid(g, xsub=1)
    t = batch._tols(tols)
    if cell_factors is None:
        f = halo_cell_factor(u, base, float(t.max()))
        cell_factors = sorted({0.8, 1.0, 1.25} |
                              ({round(f * k, 4) for k in (1.0, 1.12, 1.25, 1.5)} if f else set()))
    out = torch.empty((u.shape[0], len(t)), dtype=torch.int32, device=g.device)
    table = []
    for f in cell_factors:
        for xs in xsubs:
            grid = batch.GvecGrid(g, cell=base.cs * f, xsub=xs)
            if grid.xsub != xs:
                continue  # over the cell budget
            bins_ok = float(t.max()) < batch.BINS_TOL_LIMIT and batch.bins_fit(grid)
            methods = ["bins", "walk"] if method is None else [method]
            for m in methods:
                if m == "bins" and not bins_ok:
                    continue
                ws = batch.BinsWorkspace(u.shape[0], grid, batch.bins_box_estimate(
                    u, grid, float(t.max()))) if m == "bins" else None
                ms = _time(lambda: batch.score_grid(u, grid, t, out=out, method=m,
                                                    workspace=ws), reps)
                table.append(((f, xs, m), ms))
                del ws
            del grid
    best = min(table, key=lambda x: x[1])[0]
    _cache[grid_key(g.shape[0])] = list(best)
    _autosave()
    return best[:2], table


def grid_shape(n):
    """The tuned (cell factor, xsub) for this many g-vectors, or None."""
    if not _cache:
        return None
    t = _cache.get(grid_key(n))
    return tuple(t[:2]) if t else None


def grid_method(n):
    """The tuned score_grid method ("bins" or "walk") for this many
    g-vectors, or None."""
    t = _cache.get(grid_key(n)) if _cache else None
    return t[2] if t and len(t) > 2 else None


def save(path):
    with open(path, "w") as f:
        json.dump(_cache, f, indent=1, sort_keys=True)


def load(path):
    with open(path) as f:
        _cache.update(json.load(f))


def clear():
    _cache.clear()


def _autosave():
    p = os.environ.get(CACHE_ENV)
    if p:
        save(p)


if os.environ.get(CACHE_ENV) and os.path.exists(os.environ[CACHE_ENV]):
    load(os.environ[CACHE_ENV])
