"""Differentiable residuals of assigned peaks: grain + detector-geometry refinement.

ImageD11 refines detector geometry derivative-free: Nelder-Mead over a
goodness of fit that recomputes g-vectors and calls score_and_refine per grain
(ImageD11/refinegrains.py:517-624).  Here the same forward model --
compute_xlylzl (ImageD11/transform.py:85-147, src/cdiffraction.c:190-224),
compute_gv (src/cdiffraction.c:112-168) and the residual UBI.g - h of each
assigned peak -- has a hand-written adjoint in CUDA (csrc/adjoint.cu) behind
``torch.autograd.Function``, so gradients with respect to every UBI and to the
geometry parameters

    distance, y_center, z_center, tilt_x, tilt_y, tilt_z, wavelength, wedge,
    chi, t_x, t_y, t_z                       (ImageD11 parameter names)

come from one forward and one reverse pass over the peaks, in FP64.  The small
dense maps from those parameters to the detector matrix r = R(tilts).flip and
the chi.wedge matrix M are written in torch so autograd chains through them.

:func:`refine_geometry` minimises the residuals over the geometry with the
UBIs eliminated in closed form (each grain's least-squares UBI for the current
g-vectors, an FP64 3x3 solve), using L-BFGS on the adjoint gradient.
"""
import math

import numpy as np

from ._lib import lib, check

PARAMS = ("distance", "y_center", "z_center", "tilt_x", "tilt_y", "tilt_z", "wavelength",
          "wedge", "chi", "t_x", "t_y", "t_z")

# typical magnitudes of a useful step, used to scale the optimiser's variables
SCALES = dict(distance=100.0, y_center=1.0, z_center=1.0, tilt_x=1e-3, tilt_y=1e-3,
              tilt_z=1e-3, wavelength=1e-5, wedge=1e-2, chi=1e-2, t_x=1.0, t_y=1.0, t_z=1.0)


def _torch():
    import torch
    return torch


def detector_matrix(tilt_x, tilt_y, tilt_z, flip):
    """R3(tilt_x).R2(tilt_y).R1(tilt_z).flip (ImageD11/transform.py:51-82,
    :688-692), differentiable in the tilts (radians)."""
    torch = _torch()
    z = torch.zeros((), dtype=torch.float64, device=tilt_x.device)
    o = torch.ones((), dtype=torch.float64, device=tilt_x.device)
    cz, sz = torch.cos(tilt_z), torch.sin(tilt_z)
    cy, sy = torch.cos(tilt_y), torch.sin(tilt_y)
    cx, sx = torch.cos(tilt_x), torch.sin(tilt_x)
    r1 = torch.stack([torch.stack([cz, -sz, z]), torch.stack([sz, cz, z]),
                      torch.stack([z, z, o])])
    r2 = torch.stack([torch.stack([cy, z, sy]), torch.stack([z, o, z]),
                      torch.stack([-sy, z, cy])])
    r3 = torch.stack([torch.stack([o, z, z]), torch.stack([z, cx, -sx]),
                      torch.stack([z, sx, cx])])
    return r3 @ r2 @ r1 @ flip


def wedgechi_matrix(wedge, chi):
    """The chi.wedge matrix M of src/cdiffraction.c:117-142, wedge and chi in
    degrees, differentiable."""
    torch = _torch()
    z = torch.zeros((), dtype=torch.float64, device=wedge.device)
    o = torch.ones((), dtype=torch.float64, device=wedge.device)
    w = wedge * (math.pi / 180.0)
    c = chi * (math.pi / 180.0)
    sw, cw, sc, cc = torch.sin(w), torch.cos(w), torch.sin(c), torch.cos(c)
    W = torch.stack([torch.stack([cw, z, -sw]), torch.stack([z, o, z]),
                     torch.stack([sw, z, cw])])
    C = torch.stack([torch.stack([o, z, z]), torch.stack([z, cc, -sc]),
                     torch.stack([z, sc, cc])])
    return W @ C


class PeakTable:
    """Assigned peaks stored grain by grain, resident on the GPU.

    sc, fc, omega: (n,) detector slow/fast pixel positions and omega (deg);
    hkl: (n,3) the assigned integer indices; offsets: (ngrains+1,) so grain G
    owns peaks offsets[G]..offsets[G+1]-1.  Fixed detector constants
    (pixel sizes, flip o11..o22, omegasign) come from ``geo`` (a dict with
    ImageD11 parameter names)."""

    def __init__(self, sc, fc, omega, hkl, offsets, geo):
        torch = _torch()
        dev = "cuda"

        def f64(a):
            if torch.is_tensor(a):
                return a.to(dev, torch.float64).contiguous()
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

        self.sc, self.fc, self.omega = f64(sc), f64(fc), f64(omega)
        self.hkl = f64(hkl).reshape(-1, 3)
        if torch.is_tensor(offsets):
            offsets = offsets.cpu().numpy()
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        self.offsets = torch.as_tensor(off, device=dev)
        self.ngrains = len(off) - 1
        self.n = int(off[-1]) if len(off) else 0
        self.y_size = float(geo["y_size"])
        self.z_size = float(geo["z_size"])
        self.omegasign = float(geo["omegasign"])
        self.flip = torch.tensor([[1.0, 0.0, 0.0], [0.0, geo["o22"], geo["o21"]],
                                  [0.0, geo["o12"], geo["o11"]]], dtype=torch.float64,
                                 device=dev)
        self.ws = torch.empty(lib.id11b_adjoint_workspace_bytes(max(self.ngrains, 1)) // 8,
                              dtype=torch.float64, device=dev)


def _geom_host(r, M, t, lam, dist, yc, zc, peaks):
    g = np.empty(28)
    g[0:9] = r.detach().cpu().numpy().ravel()
    g[9:18] = M.detach().cpu().numpy().ravel()
    g[18:21] = t.detach().cpu().numpy()
    g[21] = float(lam)
    g[22] = float(dist)
    g[23] = float(yc)
    g[24] = float(zc)
    g[25] = peaks.y_size
    g[26] = peaks.z_size
    g[27] = peaks.omegasign
    return g


def _stream():
    return _torch().cuda.current_stream().cuda_stream


class _Residuals(_torch().autograd.Function):
    """res (n,3) = UBI_G . g(r, M, t, wavelength, distance, centres) - hkl."""

    @staticmethod
    def forward(ctx, r, M, t, lam, dist, yc, zc, ubis, peaks):
        torch = _torch()
        geom = _geom_host(r, M, t, lam, dist, yc, zc, peaks)
        u = ubis.detach().reshape(-1, 9).contiguous()
        res = torch.empty((peaks.n, 3), dtype=torch.float64, device=u.device)
        ssq = torch.empty(max(peaks.ngrains, 1), dtype=torch.float64, device=u.device)
        check(lib.id11b_dev_residuals(geom.ctypes.data, peaks.sc.data_ptr(), peaks.fc.data_ptr(),
                                      peaks.omega.data_ptr(), peaks.hkl.data_ptr(),
                                      peaks.offsets.data_ptr(), u.data_ptr(), peaks.ngrains,
                                      res.data_ptr(), None, ssq.data_ptr(), _stream()),
              "residuals")
        ctx.peaks = peaks
        ctx.geom = geom
        ctx.save_for_backward(r, u)
        ctx.ubi_shape = ubis.shape
        return res

    @staticmethod
    def backward(ctx, grad_res):
        torch = _torch()
        r, u = ctx.saved_tensors
        peaks = ctx.peaks
        gr = grad_res.detach().to(torch.float64).contiguous()
        gu = torch.empty_like(u)
        gl = torch.empty(22, dtype=torch.float64, device=u.device)
        check(lib.id11b_dev_residuals_adjoint(
            ctx.geom.ctypes.data, peaks.sc.data_ptr(), peaks.fc.data_ptr(),
            peaks.omega.data_ptr(), peaks.hkl.data_ptr(), peaks.offsets.data_ptr(),
            u.data_ptr(), peaks.ngrains, gr.data_ptr(), gu.data_ptr(), gl.data_ptr(),
            peaks.ws.data_ptr(), peaks.ws.numel() * 8, _stream()), "residuals_adjoint")
        dM = gl[0:9].view(3, 3)
        dlam = gl[9]
        dt = gl[10:13]
        A = gl[13:16]
        dr = torch.zeros((3, 3), dtype=torch.float64, device=u.device)
        dr[:, 1] = gl[16:19]
        dr[:, 2] = gl[19:22]
        ddist = A[0]
        dyc = -peaks.y_size * torch.dot(r.detach()[:, 1], A)
        dzc = -peaks.z_size * torch.dot(r.detach()[:, 2], A)
        return dr, dM, dt, dlam, ddist, dyc, dzc, gu.view(ctx.ubi_shape), None


def residuals(params, ubis, peaks):
    """Residuals (n,3) of every assigned peak, differentiable with respect to
    ``params`` -- a (12,) float64 CUDA tensor in the order of PARAMS -- and
    ``ubis`` -- (ngrains,3,3) float64 CUDA tensor."""
    dist, yc, zc, tx, ty, tz, lam, wedge, chi, t0, t1, t2 = params.unbind(0)
    r = detector_matrix(tx, ty, tz, peaks.flip)
    M = wedgechi_matrix(wedge, chi)
    t = _torch().stack([t0, t1, t2])
    return _Residuals.apply(r, M, t, lam, dist, yc, zc, ubis, peaks)


def params_tensor(geo):
    """(12,) float64 CUDA tensor of the PARAMS entries of an ImageD11-style dict."""
    torch = _torch()
    return torch.tensor([float(geo[k]) for k in PARAMS], dtype=torch.float64, device="cuda")


def gvectors(params, peaks):
    """g-vectors (n,3) of the peaks for the geometry ``params`` (no gradient)."""
    torch = _torch()
    with torch.no_grad():
        dist, yc, zc, tx, ty, tz, lam, wedge, chi, t0, t1, t2 = params.detach().unbind(0)
        r = detector_matrix(tx, ty, tz, peaks.flip)
        M = wedgechi_matrix(wedge, chi)
        t = torch.stack([t0, t1, t2])
        geom = _geom_host(r, M, t, lam, dist, yc, zc, peaks)
        dev = peaks.sc.device
        zero = torch.zeros((max(peaks.ngrains, 1), 9), dtype=torch.float64, device=dev)
        res = torch.empty((peaks.n, 3), dtype=torch.float64, device=dev)
        g = torch.empty((peaks.n, 3), dtype=torch.float64, device=dev)
        ssq = torch.empty(max(peaks.ngrains, 1), dtype=torch.float64, device=dev)
        check(lib.id11b_dev_residuals(geom.ctypes.data, peaks.sc.data_ptr(), peaks.fc.data_ptr(),
                                      peaks.omega.data_ptr(), peaks.hkl.data_ptr(),
                                      peaks.offsets.data_ptr(), zero.data_ptr(), peaks.ngrains,
                                      res.data_ptr(), g.data_ptr(), ssq.data_ptr(), _stream()),
              "gvectors")
    return g


def best_ubis(g, peaks):
    """Each grain's UBI minimising sum |UBI.g - h|^2 over its peaks:
    UBI = (sum h g^T)(sum g g^T)^-1, an FP64 3x3 solve per grain."""
    torch = _torch()
    sizes = peaks.offsets[1:] - peaks.offsets[:-1]
    gi = torch.repeat_interleave(torch.arange(peaks.ngrains, device=g.device), sizes)
    h = peaks.hkl
    A = torch.zeros((peaks.ngrains, 3, 3), dtype=torch.float64, device=g.device)
    B = torch.zeros_like(A)
    A.index_add_(0, gi, h[:, :, None] * g[:, None, :])
    B.index_add_(0, gi, g[:, :, None] * g[:, None, :])
    return torch.linalg.solve(B, A.transpose(1, 2)).transpose(1, 2).contiguous()


def loss(params, ubis, peaks):
    """0.5 * sum of squared residuals (differentiable)."""
    r = residuals(params, ubis, peaks)
    return 0.5 * (r * r).sum()


def refine_geometry(peaks, params0, free=None, max_iter=60, history=20):
    """Refine the geometry by L-BFGS with every grain's UBI re-solved in closed
    form at each evaluation (variable projection: at the best UBIs the loss
    gradient with respect to the geometry is the partial derivative, which the
    adjoint gives).  ``free``: names of the parameters to refine (default: all
    but wavelength, which the free UBIs make unidentifiable -- a common scale
    of g and of every UBI leaves the residuals unchanged).  When every grain
    sits at the one translation t, two more directions are flat: t_z moves the
    spots as a z_center shift does (the omega axis is z) and tilt_x trades
    against chi (both rotate about the beam); the optimiser then settles
    anywhere along them, which leaves the residuals, the other parameters and
    the combinations z_center*z_size + t_z and tilt_x - chi (radians) fixed.
    Returns (params, ubis, history of loss values)."""
    torch = _torch()
    free = [p for p in PARAMS if p != "wavelength"] if free is None else list(free)
    mask = torch.tensor([p in free for p in PARAMS], dtype=torch.float64, device="cuda")
    scale = torch.tensor([SCALES[p] for p in PARAMS], dtype=torch.float64, device="cuda")
    base = params0.detach().to(torch.float64).clone()
    x = torch.zeros(len(PARAMS), dtype=torch.float64, device="cuda", requires_grad=True)
    hist = []

    def current():
        return base + mask * scale * x

    def closure():
        opt.zero_grad()
        p = current()
        u = best_ubis(gvectors(p, peaks), peaks)
        value = loss(p, u, peaks)
        value.backward()
        hist.append(float(value.detach()))
        return value

    opt = torch.optim.LBFGS([x], lr=1.0, max_iter=max_iter, history_size=history,
                            tolerance_grad=1e-14, tolerance_change=1e-16,
                            line_search_fn="strong_wolfe")
    opt.step(closure)
    p = current().detach()
    return p, best_ubis(gvectors(p, peaks), peaks), hist
