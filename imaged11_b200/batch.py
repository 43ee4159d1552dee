"""Batched grain scoring and refinement on the GPU (beyond the per-call drop-in).

The reference scores trial orientations one ``score`` call at a time
(ImageD11/indexing.py:762-874, ``indexer.scorethem``) and refines grains one
``score_and_refine`` call at a time (ImageD11/refinegrains.py:459-498).  These
functions run whole batches in one launch sequence with identical
assignments:

* :class:`GvecSet` keeps a g-vector table resident on the GPU in FP64 plus the
  FP32 float4 copy and screening metadata the batched kernels read;
* :func:`score_batch` -- counts (and drlv2 sums) for M UBIs x T tolerances,
  FP32 screening with exact FP64 recheck inside a proven error band;
* :func:`score_many_fp64` -- the same counts from the plain FP64 kernel
  (reference arithmetic, one thread per g), the baseline;
* :func:`refine_batch` -- ``iters`` score_and_refine rounds for M UBIs against
  all g-vectors.

All tensors live on the current CUDA device; work is enqueued on the current
stream.
"""
import numpy as np

from ._lib import lib, check

ID11B_ERR_SIZE = 4


def _torch():
    import torch
    return torch


def _stream():
    return _torch().cuda.current_stream().cuda_stream


def _dev(a, dtype):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            a = a.cuda()
        return a.to(dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dtype).contiguous()


def _tols(tols):
    t = np.ascontiguousarray(np.atleast_1d(tols), dtype=np.float64)
    if t.ndim != 1 or not 1 <= len(t) <= 4:
        raise ValueError("between 1 and 4 tolerances are supported per launch")
    return t


class GvecSet:
    """g-vectors (n,3) float64 resident on the GPU with their FP32 copy.

    ``gv`` may be a numpy array or a CUDA tensor; it is copied once."""

    def __init__(self, gv):
        torch = _torch()
        self.gv = _dev(gv, torch.float64).reshape(-1, 3)
        self.n = self.gv.shape[0]
        self.g4 = torch.empty((max(self.n, 1), 4), dtype=torch.float32, device=self.gv.device)
        wsb = lib.id11b_gvec_workspace_bytes(self.n)
        self.ws = torch.empty(wsb, dtype=torch.uint8, device=self.gv.device)
        self.prepare()

    def prepare(self):
        """(Re)build the FP32 copy and screening data from self.gv."""
        check(lib.id11b_dev_prepare_gvecs(self.gv.data_ptr(), self.n, self.g4.data_ptr(),
                                          self.ws.data_ptr(), self.ws.numel(), _stream()),
              "prepare_gvecs")


class BatchWorkspace:
    """Reusable scratch for score_batch / refine_batch of a given size."""

    def __init__(self, m, n, refine=False):
        torch = _torch()
        self.m, self.n, self.refine = m, n, int(bool(refine))
        wsb = lib.id11b_batch_workspace_bytes(m, n, self.refine)
        self.buf = torch.empty(wsb, dtype=torch.uint8, device="cuda")

    def fits(self, m, n, refine):
        return lib.id11b_batch_workspace_bytes(m, n, int(bool(refine))) <= self.buf.numel()

    def stats(self):
        """(FP64 re-evaluations, UBIs evaluated wholly in FP64); raises on a
        device error flag.  Synchronises the stream."""
        import ctypes
        nr = ctypes.c_int64(0)
        nf = ctypes.c_int32(0)
        er = ctypes.c_int32(0)
        rc = lib.id11b_batch_stats(self.buf.data_ptr(), self.m, self.n, self.refine,
                                   ctypes.addressof(nr), ctypes.addressof(nf),
                                   ctypes.addressof(er), _stream())
        check(rc, "batch")
        return nr.value, nf.value


def score_batch(ubis, gvs, tols, sums=False, workspace=None, out=None, tile=None):
    """Counts of g-vectors indexed by each UBI at each tolerance.

    ubis: (m,3,3) float64 (numpy or CUDA); gvs: GvecSet; tols: 1-4 values.
    Returns an int32 CUDA tensor (m, len(tols)) -- and, with sums=True, the
    float64 tensor of summed drlv2 of the counted pairs.
    tile: (UBIs per thread, gsplit) launch shape; None takes the shape
    tune.tune_score found for this size, else the built-in heuristic."""
    torch = _torch()
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    m = u.shape[0]
    t = _tols(tols)
    ws = workspace if workspace is not None and workspace.fits(m, gvs.n, False) else \
        BatchWorkspace(m, gvs.n, False)
    counts = out if out is not None else torch.empty((m, len(t)), dtype=torch.int32,
                                                     device=u.device)
    s = torch.empty((m, len(t)), dtype=torch.float64, device=u.device) if sums else None
    if tile is None:
        from . import tune
        tile = tune.score_tile(m, gvs.n, len(t)) or (0, 0)
    check(lib.id11b_dev_score_batch_tiled(u.data_ptr(), m, gvs.gv.data_ptr(),
                                          gvs.g4.data_ptr(), gvs.n, gvs.ws.data_ptr(),
                                          t.ctypes.data, len(t), counts.data_ptr(),
                                          s.data_ptr() if sums else None, int(tile[0]),
                                          int(tile[1]), ws.buf.data_ptr(), ws.buf.numel(),
                                          _stream()),
          "score_batch")
    score_batch.last_workspace = ws
    return (counts, s) if sums else counts


class GvecGrid:
    """Reciprocal-space cell index of a set of g-vectors, for score_grid.

    gv: (n,3) float64 (numpy or CUDA) or a GvecSet.  cell: side of the cells
    in y and z in 1/Angstrom (None: about one g per cell of the bounding
    cube); xsub: x cells per y/z cell side.  Finer x cells shorten the scanned
    rows at the cost of memory: on B200 with 1.1M g, 20,000 UBIs scored in
    8.2 / 7.5 / 7.4 / 7.2 ms at xsub 1 / 2 / 4 / 8.  By default xsub is capped so
    the cell-start table stays near 32 MB (in L2).  Building reads two numbers
    back to the host (the bounds that size the grid); scoring does not."""

    XSUB = 8
    MAX_CELLS = 1 << 23

    def __init__(self, gv, cell=None, xsub=None):
        import ctypes
        torch = _torch()
        g = gv.gv if isinstance(gv, GvecSet) else _dev(gv, torch.float64).reshape(-1, 3)
        self.gv = g.contiguous()
        self.n = self.gv.shape[0]
        dev = self.gv.device
        bounds = torch.zeros(2, dtype=torch.int32, device=dev)
        check(lib.id11b_dev_gvec_bounds(self.gv.data_ptr(), self.n, bounds.data_ptr(),
                                        _stream()), "gvec_bounds")
        b = bounds.cpu().numpy().view(np.float32)
        self.gmax, self.rmax = float(b[0]), float(b[1])
        nx = ctypes.c_int32(0)
        cs = ctypes.c_double(0.)
        if cell is None and xsub is None:  # a shape tune.tune_grid found for this size
            from . import tune
            shape = tune.grid_shape(self.n)
            if shape:
                check(lib.id11b_grid_plan(self.gmax, self.n, 0., ctypes.addressof(nx),
                                          ctypes.addressof(cs)), "grid_plan")
                cell, xsub = cs.value * shape[0], int(shape[1])
        check(lib.id11b_grid_plan(self.gmax, self.n, float(cell or 0.), ctypes.addressof(nx),
                                  ctypes.addressof(cs)), "grid_plan")
        self.nx, self.cs = nx.value, cs.value
        if xsub is None:
            xsub = max(1, min(self.XSUB, self.MAX_CELLS // self.nx ** 3))
        self.xsub = max(1, min(int(xsub), 16, (1 << 26) // self.nx ** 3))
        nbytes = lib.id11b_grid_bytes(self.n, self.nx, self.xsub)
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        check(lib.id11b_dev_build_grid(self.gv.data_ptr(), self.n, self.gmax, self.rmax,
                                       self.cs, self.nx, self.xsub, self.buf.data_ptr(), nbytes,
                                       _stream()), "build_grid")

    def refresh(self):
        """Rebuild the index from self.gv (changed in place) into the same
        buffer and shape, reading nothing back.  g that left the cube and ball
        the index was sized for (|g_j| <= gmax, |g| <= rmax) go to the list of
        g scored by a plain scan, as non-finite ones do: counts stay exact,
        and a rebuild with fresh bounds restores the speed."""
        check(lib.id11b_dev_build_grid(self.gv.data_ptr(), self.n, self.gmax, self.rmax,
                                       self.cs, self.nx, self.xsub, self.buf.data_ptr(),
                                       self.buf.numel(), _stream()), "build_grid")

    def stats(self):
        """dict: regular / listed g-vectors; UBIs scanned plainly and pairs
        evaluated by the last score_grid call (synchronises)."""
        import ctypes
        v = [ctypes.c_int64(0) for _ in range(5)]
        check(lib.id11b_grid_stats(self.buf.data_ptr(), *[ctypes.addressof(x) for x in v],
                                   _stream()), "grid_stats")
        return dict(zip(("regular", "special", "fallback_ubis", "pairs_tested",
                         "pairs_screened"), (x.value for x in v)))


BINS_TOL_LIMIT = 0.4   # the binned join takes tolerances below this
BINS_MAX_BOXES = 1 << 29   # default workspace cap (4 GiB of boxes); more run in UBI ranges
BINS_MAX_ROWS = 65536      # the binned join holds nx^2 rows of cells ...
BINS_MAX_XCELLS = 8191     # ... and nx * xsub x cells per row


def bins_fit(grid):
    """Whether the binned join takes this grid's shape."""
    return grid.nx * grid.nx <= BINS_MAX_ROWS and grid.nx * grid.xsub <= BINS_MAX_XCELLS


def bins_box_estimate(ubis, grid, tmax):
    """An estimate (about 25 % above the expected count) of the (UBI, hkl)
    boxes the binned join enumerates for these UBIs: the lattice points of
    each UBI within rmax + |w| of the origin.  Reads one number back."""
    torch = _torch()
    u = _dev(ubis, torch.float64).reshape(-1, 3, 3)
    if u.shape[0] == 0:
        return 0
    det = torch.nan_to_num(torch.linalg.det(u).abs(), nan=0.0, posinf=0.0)
    ok = det > 0
    ub = torch.linalg.inv(torch.where(ok[:, None, None], u, torch.eye(3, dtype=u.dtype,
                                                                    device=u.device)))
    w = (tmax + 1e-6) * ub.norm(dim=2).norm(dim=1)
    r = grid.rmax + torch.nan_to_num(w, nan=0.0, posinf=0.0)
    est = (4.0 / 3.0 * np.pi) * (r ** 3) * det * ok
    # a UBI with more candidate hkl than g-vectors, or a large row sum, is
    # scanned plainly and enumerates no boxes
    est = torch.where(est <= grid.n, est, torch.zeros_like(est))
    total = 1.25 * float(est.sum().item()) + 64 * u.shape[0]
    return int(min(total, BINS_MAX_BOXES))


class BinsWorkspace:
    """Reusable scratch of the binned join for m UBIs on a grid, holding
    `boxes` (UBI, hkl) boxes at a time (a shorter workspace still works: the
    UBIs are then processed in ranges that fit)."""

    def __init__(self, m, grid, boxes):
        torch = _torch()
        self.m, self.nx, self.xsub, self.boxes = m, grid.nx, grid.xsub, int(boxes)
        nbytes = lib.id11b_grid_bins_workspace_bytes(m, grid.nx, grid.xsub, self.boxes)
        if nbytes < 0:
            raise ValueError("bad binned-join workspace size")
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=grid.gv.device)

    def fits(self, m, grid, boxes):
        return lib.id11b_grid_bins_workspace_bytes(m, grid.nx, grid.xsub, int(boxes)) <= \
            self.buf.numel()


def score_grid(ubis, grid, tols, sums=False, workspace=None, out=None, method=None):
    """score_batch through the cell index: the same counts (and, with
    sums=True, FP64 sums of the counted drlv2) for every UBI and tolerance,
    testing only the g-vectors near each UB.hkl.  grid: GvecGrid.

    method "bins": the binned join, every (UBI, hkl) box against the g of its
    bin's region in FP32 with the proven FP64 recheck band (tolerances below
    0.4; its FP64 sums accumulated in fixed point, reproducible); "walk":
    per-box lookups with every candidate evaluated in FP64 (any tolerance,
    sums in a fixed order).  Both give the same counts.  None: the method
    tune.tune_grid found fastest for this many g-vectors, else "bins" where it
    applies.  workspace: a BinsWorkspace ("bins") or a uint8 CUDA tensor
    ("walk")."""
    torch = _torch()
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    m = u.shape[0]
    t = _tols(tols)
    auto = method is None
    if auto:
        from . import tune
        bins_ok = float(t.max()) < BINS_TOL_LIMIT and bins_fit(grid)
        method = "bins" if bins_ok and tune.grid_method(grid.n) != "walk" else "walk"
    elif method == "bins" and not bins_fit(grid):
        raise ValueError("the binned join holds at most %d rows of %d x cells; use "
                         "method='walk' or coarser cells" % (BINS_MAX_ROWS, BINS_MAX_XCELLS))
    counts = out if out is not None else torch.empty((m, len(t)), dtype=torch.int32,
                                                     device=u.device)
    s = torch.empty((m, len(t)), dtype=torch.float64, device=u.device) if sums else None
    if method == "bins":
        ws = workspace if isinstance(workspace, BinsWorkspace) and workspace.m >= m and \
            (workspace.nx, workspace.xsub) == (grid.nx, grid.xsub) else None
        if ws is None:
            ws = BinsWorkspace(m, grid, bins_box_estimate(u, grid, float(t.max())))
        rc = lib.id11b_dev_score_grid_bins(u.data_ptr(), m, grid.gv.data_ptr(), grid.n,
                                           grid.nx, grid.xsub, grid.buf.data_ptr(),
                                           t.ctypes.data, len(t), counts.data_ptr(),
                                           s.data_ptr() if sums else None, ws.buf.data_ptr(),
                                           ws.buf.numel(), _stream())
        score_grid.last_workspace = ws
        if not (auto and rc == ID11B_ERR_SIZE):   # cells far smaller than the boxes: walk
            check(rc, "score_grid_bins")
            return (counts, s) if sums else counts
        method = "walk"
    if method != "walk":
        raise ValueError("method: 'bins' or 'walk'")
    need = lib.id11b_grid_score_workspace_bytes(m, len(t))
    ws = workspace if workspace is not None and not isinstance(workspace, BinsWorkspace) and \
        workspace.numel() >= need else torch.empty(need, dtype=torch.uint8, device=u.device)
    check(lib.id11b_dev_score_grid(u.data_ptr(), m, grid.gv.data_ptr(), grid.n, grid.nx,
                                   grid.xsub, grid.buf.data_ptr(), t.ctypes.data, len(t), counts.data_ptr(),
                                   s.data_ptr() if sums else None, ws.data_ptr(), ws.numel(),
                                   _stream()), "score_grid")
    return (counts, s) if sums else counts


def refine_grid(ubis, grid, tol, iters=1):
    """``iters`` rounds of score_and_refine for every UBI against every g,
    through the cell index (the result of refine_batch, found by lookup).
    Returns (ubis (m,3,3) refined, npk, mean drlv2 of the last round's input
    UBIs) as CUDA tensors; a CUDA float64 input is updated in place."""
    torch = _torch()
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    m = u.shape[0]
    npk = torch.empty(m, dtype=torch.int32, device=u.device)
    mean = torch.empty(m, dtype=torch.float64, device=u.device)
    ws = torch.empty(max(lib.id11b_grid_refine_workspace_bytes(m), 256), dtype=torch.uint8,
                     device=u.device)
    check(lib.id11b_dev_refine_grid(u.data_ptr(), m, grid.gv.data_ptr(), grid.n, grid.nx,
                                    grid.xsub, grid.buf.data_ptr(), float(tol), int(iters),
                                    npk.data_ptr(), mean.data_ptr(), ws.data_ptr(), ws.numel(),
                                    _stream()), "refine_grid")
    return u.view(-1, 3, 3), npk, mean


def score_and_assign_grid(ubis, grid, tol, drlv2, labels, grain_labels=None, npk=False,
                          method="walk", workspace=None):
    """score_and_assign (ImageD11 src/closest.c:366-397) for every grain in
    order, as ImageD11/indexing.py fight_over_peaks calls it, in one pass
    over the cell index: drlv2 (n float64) and labels (n int32) -- CUDA
    tensors, or numpy arrays copied back in place -- end up exactly as after
    the sequential calls score_and_assign(ubis[i], gv, tol, drlv2, labels,
    grain_labels[i]).  grain_labels: strictly increasing ints (default
    0 .. m-1).  With npk=True also returns the int32 count of peaks holding
    each grain's label at the end.  method: "walk" looks up the g near each
    grain's lattice points; "bins" takes the pairs from the binned join (tol
    below 0.4, the grid within the join's limits; workspace: a BinsWorkspace
    to reuse) -- the same result."""
    torch = _torch()
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    m = u.shape[0]
    dev = u.device
    host = isinstance(drlv2, np.ndarray)
    if host != isinstance(labels, np.ndarray):
        raise TypeError("drlv2 and labels: both numpy or both CUDA tensors")
    if host:
        if drlv2.dtype != np.float64 or labels.dtype != np.int32:
            raise TypeError("drlv2 must be float64 and labels int32")
        d = torch.as_tensor(drlv2).to(dev)
        lab = torch.as_tensor(labels).to(dev)
    else:
        if drlv2.dtype != torch.float64 or labels.dtype != torch.int32:
            raise TypeError("drlv2 must be float64 and labels int32")
        d, lab = drlv2, labels
    if d.numel() != grid.n or lab.numel() != grid.n or not (d.is_contiguous() and
                                                           lab.is_contiguous()):
        raise ValueError("drlv2 and labels need one contiguous entry per g-vector")
    gl = None
    if grain_labels is not None:
        gl = torch.as_tensor(np.asarray(grain_labels, dtype=np.int32)).to(dev) \
            if not torch.is_tensor(grain_labels) else grain_labels.to(dev, torch.int32)
        if gl.numel() != m:
            raise ValueError("one grain label per UBI")
        if m > 1 and not bool((gl[1:] > gl[:-1]).all()):
            raise ValueError("grain_labels must be strictly increasing")
        gl = gl.contiguous()
    counts = torch.empty(m, dtype=torch.int32, device=dev) if npk else None
    if method == "bins":
        if not (float(tol) < BINS_TOL_LIMIT and bins_fit(grid)):
            raise ValueError("method='bins' needs tol < %g and a grid within the join's "
                             "limits" % BINS_TOL_LIMIT)
        # a caller's workspace of this shape is used whatever it holds (the
        # grains then run in ranges of boxes that fit), as in score_grid
        bws = workspace if isinstance(workspace, BinsWorkspace) and workspace.m >= m and \
            (workspace.nx, workspace.xsub) == (grid.nx, grid.xsub) else \
            BinsWorkspace(m, grid, bins_box_estimate(u, grid, float(tol)))
        best = torch.empty(grid.n, dtype=torch.int64, device=dev)
        win = torch.empty(grid.n, dtype=torch.int32, device=dev)
        args = (u.data_ptr(), m)
        shape = (grid.n, grid.nx, grid.xsub, grid.buf.data_ptr(), float(tol))
        check(lib.id11b_dev_assign_grid_pass(*args, 0, *shape, d.data_ptr(), -1, best.data_ptr(),
                                             win.data_ptr(), _stream()), "assign_pass")
        check(lib.id11b_dev_assign_grid_bins(*args, grid.gv.data_ptr(), *shape, d.data_ptr(),
                                             best.data_ptr(), win.data_ptr(), bws.buf.data_ptr(),
                                             bws.buf.numel(), _stream()), "assign_grid_bins")
        check(lib.id11b_dev_assign_grid_final(*args, gl.data_ptr() if gl is not None else None,
                                              grid.gv.data_ptr(), *shape, best.data_ptr(),
                                              win.data_ptr(), d.data_ptr(), lab.data_ptr(),
                                              counts.data_ptr() if npk else None, _stream()),
              "assign_final")
        if host:
            drlv2[:] = d.cpu().numpy()
            labels[:] = lab.cpu().numpy()
        return counts
    if method != "walk":
        raise ValueError("method: 'walk' or 'bins'")
    ws = torch.empty(lib.id11b_assign_workspace_bytes(grid.n), dtype=torch.uint8, device=dev)
    check(lib.id11b_dev_score_and_assign_grid(u.data_ptr(), m,
                                              gl.data_ptr() if gl is not None else None,
                                              grid.gv.data_ptr(), grid.n, grid.nx, grid.xsub,
                                              grid.buf.data_ptr(), float(tol), d.data_ptr(),
                                              lab.data_ptr(),
                                              counts.data_ptr() if npk else None,
                                              ws.data_ptr(), ws.numel(), _stream()),
          "score_and_assign_grid")
    if host:
        drlv2[:] = d.cpu().numpy()
        labels[:] = lab.cpu().numpy()
    return counts


def score_many_fp64(ubis, gv, tols, out=None):
    """Plain FP64 batched score (reference arithmetic).  gv: (n,3) float64 CUDA
    tensor or GvecSet.  Returns int32 (m, len(tols))."""
    torch = _torch()
    g = gv.gv if isinstance(gv, GvecSet) else _dev(gv, torch.float64).reshape(-1, 3)
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    t = _tols(tols)
    counts = out if out is not None else torch.empty((u.shape[0], len(t)), dtype=torch.int32,
                                                     device=u.device)
    check(lib.id11b_dev_score_many_fp64(u.data_ptr(), u.shape[0], g.data_ptr(), g.shape[0],
                                        t.ctypes.data, len(t), counts.data_ptr(), _stream()),
          "score_many_fp64")
    return counts


def refine_batch(ubis, gvs, tol, iters=1, workspace=None):
    """``iters`` rounds of score_and_refine for every UBI against every g.

    ubis: (m,3,3) float64 CUDA tensor, refined in place (a numpy array is
    copied to the GPU and the refined copy returned).  Returns
    (ubis, npk, mean_drlv2) of the last round."""
    torch = _torch()
    if isinstance(ubis, torch.Tensor) and ubis.is_cuda:
        if ubis.dtype != torch.float64 or not ubis.is_contiguous():
            raise ValueError("ubis: contiguous float64 CUDA tensor required")
        u = ubis
    else:
        u = _dev(ubis, torch.float64)
    u9 = u.view(-1, 9)
    m = u9.shape[0]
    ws = workspace if workspace is not None and workspace.fits(m, gvs.n, True) else \
        BatchWorkspace(m, gvs.n, True)
    npk = torch.zeros(m, dtype=torch.int32, device=u.device)
    mean = torch.zeros(m, dtype=torch.float64, device=u.device)
    check(lib.id11b_dev_refine_batch(u9.data_ptr(), m, gvs.gv.data_ptr(), gvs.g4.data_ptr(),
                                     gvs.n, gvs.ws.data_ptr(), float(tol), int(iters),
                                     npk.data_ptr(), mean.data_ptr(), ws.buf.data_ptr(),
                                     ws.buf.numel(), _stream()), "refine_batch")
    refine_batch.last_workspace = ws
    return u.view(-1, 3, 3), npk, mean


class GrainSet:
    """Grains with their own peaks, for per-grain refinement.

    gv: (n,3) float64 g-vectors sorted by grain; offsets: (ngrains+1,) int64 so
    grain g owns gv[offsets[g]:offsets[g+1]]; ubis: (ngrains,3,3).  Everything
    is copied to the GPU once; grains are processed largest first.

    threads: CTA size of the persistent launch; None takes the size
    tune.tune_refine found for this many grains and peaks, else 64.  Measured
    on B200 with 2,000 grains of 20..1,500 peaks: 64 threads 53 us for 5
    rounds, 128 -> 87 us, 256 -> 147 us -- many small CTAs keep more grains in
    flight, which matters more than the longest grain's share of lanes."""

    def __init__(self, gv, offsets, ubis, threads=None):
        torch = _torch()
        self.gv = _dev(gv, torch.float64).reshape(-1, 3)
        if torch.is_tensor(offsets):
            offsets = offsets.cpu().numpy()
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        self.ngrains = len(off) - 1
        dev = self.gv.device
        self.offsets = torch.as_tensor(off, device=dev)
        sizes = np.diff(off)
        self.order = torch.as_tensor(np.argsort(-sizes, kind="stable").astype(np.int32),
                                     device=dev)
        self.ubis = _dev(ubis, torch.float64).reshape(-1, 9).contiguous()
        self.npk = torch.zeros(self.ngrains, dtype=torch.int32, device=dev)
        self.mean = torch.zeros(self.ngrains, dtype=torch.float64, device=dev)
        self.ws = torch.zeros(lib.id11b_refine_csr_workspace_bytes(), dtype=torch.uint8,
                              device=dev)
        self.peaks = int(off[-1] - off[0]) if len(off) else 0
        if threads is None:
            from . import tune
            threads = tune.refine_threads(self.ngrains, self.peaks) or 64
        self.threads = int(threads)

    def refine(self, tol, iters, persistent=True, precision="fp64"):
        """Enqueue `iters` score_and_refine rounds for every grain (in place).
        persistent=False runs the plain baseline: one launch per round, one
        128-thread CTA per grain.  precision "f32c": FP32 screening with the
        proven FP64 recheck band and compensated FP32 normal-equation sums
        (FP64 3x3 solves; every |g_j| <= 1024, tol < 0.4) instead of FP64
        screening and sums -- the same accepted pairs, UBIs within ~1e-14."""
        if precision == "f32c":
            if not hasattr(self, "gmax"):
                self.gmax = float(self.gv.abs().max().item()) if self.peaks else 0.0
            check(lib.id11b_dev_refine_csr_f32c(self.ubis.data_ptr(), self.gv.data_ptr(),
                                                self.offsets.data_ptr(), self.order.data_ptr(),
                                                self.ngrains, float(tol), int(iters),
                                                self.gmax, self.npk.data_ptr(),
                                                self.mean.data_ptr(), self.ws.data_ptr(),
                                                self.ws.numel(), _stream()), "refine_csr_f32c")
        elif precision != "fp64":
            raise ValueError("precision: 'fp64' or 'f32c'")
        elif persistent:
            self._launch(tol, iters, 1, self.threads)
        else:
            for _ in range(iters):
                self._launch(tol, 1, 0, 128)
        return self.ubis.view(-1, 3, 3), self.npk, self.mean

    def _launch(self, tol, iters, persistent, threads):
        check(lib.id11b_dev_refine_csr(self.ubis.data_ptr(), self.gv.data_ptr(),
                                       self.offsets.data_ptr(), self.order.data_ptr(),
                                       self.ngrains, float(tol), int(iters), persistent,
                                       threads, self.npk.data_ptr(), self.mean.data_ptr(),
                                       self.ws.data_ptr(), self.ws.numel(), _stream()),
              "refine_csr")

    def capture(self, tol, iters):
        """A CUDA graph of one persistent launch (counter reset + kernel) running
        `iters` rounds on the current UBIs; call .replay() on the result."""
        torch = _torch()
        saved = self.ubis.clone()
        self._launch(tol, 1, 1, self.threads)   # load the kernel outside the capture
        self.ubis.copy_(saved)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._launch(tol, iters, 1, self.threads)
        return graph


def refine_translations(xyz, omega, offsets, ubis, translations, omegasign, wavelength, wedge,
                        chi, tol=1.0, iters=20, ubis_refit=False):
    """Per-grain translations minimising the objective of
    ImageD11/refinegrains.py refinepositions / gof: at each translation the
    grain's g-vectors, one score_and_refine update of its UBI from the one
    read (``ubis``), and the sum of drlv2 below tol^2 (1.0 there) at the
    updated UBI.  All grains in one launch by damped Gauss-Newton.  xyz (n,3)
    lab positions and omega (n,) sorted by grain, offsets (ngrains+1,), ubis
    (ngrains,3,3), translations (ngrains,3) starting values.  Returns
    (translations, cost, npk) as CUDA tensors -- refinegrains' gof of grain G
    is 1e6 * cost[G] / npk[G] -- plus the updated UBIs (ngrains,3,3) at the
    returned translations with ubis_refit=True; iters=0 only evaluates the
    objective."""
    torch = _torch()
    x = _dev(xyz, torch.float64).reshape(-1, 3)
    om = _dev(omega, torch.float64).reshape(-1)
    off = _dev(offsets, torch.int64).reshape(-1)
    u = _dev(ubis, torch.float64).reshape(-1, 9)
    ng = off.numel() - 1
    t = _dev(translations, torch.float64).reshape(-1, 3).clone()
    if u.shape[0] != ng or t.shape[0] != ng or x.shape[0] != om.shape[0]:
        raise ValueError("refine_translations: inconsistent sizes")
    cost = torch.empty(ng, dtype=torch.float64, device=x.device)
    npk = torch.empty(ng, dtype=torch.int32, device=x.device)
    u1 = torch.empty((ng, 3, 3), dtype=torch.float64, device=x.device) if ubis_refit else None
    check(lib.id11b_dev_refine_translations(x.data_ptr(), om.data_ptr(), off.data_ptr(), ng,
                                            u.data_ptr(), t.data_ptr(), float(omegasign),
                                            float(wavelength), float(wedge), float(chi),
                                            float(tol), int(iters), cost.data_ptr(),
                                            npk.data_ptr(),
                                            u1.data_ptr() if u1 is not None else None,
                                            _stream()), "refine_translations")
    if ubis_refit:
        return t, cost, npk, u1
    return t, cost, npk
