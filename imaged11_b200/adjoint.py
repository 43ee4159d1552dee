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

come from one forward and one reverse pass over the peaks, in FP64.  The
parameters stay on the device: each kernel builds the detector matrix
R3.R2.R1.flip and the chi.wedge matrix from them, and the backward pass
contracts dL/d(matrices) with their derivatives itself, so no step reads the
geometry on the host.

:func:`refine_geometry` minimises the residuals over the geometry with the
UBIs eliminated in closed form (each grain's least-squares UBI for the current
g-vectors, an FP64 3x3 solve in the same kernel), using L-BFGS on the adjoint
gradient: one fused kernel and one reduction per evaluation.
"""
import numpy as np

from ._lib import lib, check

PARAMS = ("distance", "y_center", "z_center", "tilt_x", "tilt_y", "tilt_z", "wavelength",
          "wedge", "chi", "t_x", "t_y", "t_z")

# typical magnitudes of a useful step, used to scale the optimiser's variables
SCALES = dict(distance=100.0, y_center=1.0, z_center=1.0, tilt_x=1e-3, tilt_y=1e-3,
              tilt_z=1e-3, wavelength=1e-5, wedge=1e-2, chi=1e-2, t_x=1.0, t_y=1.0, t_z=1.0)

# fixed detector constants, in the order the kernels take them
DETECTOR = ("y_size", "z_size", "omegasign", "o11", "o12", "o21", "o22")


def _torch():
    import torch
    return torch


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
        # host copy of the fixed constants, read by each call
        self.det = np.array([float(geo[k]) for k in DETECTOR], dtype=np.float64)
        self.ws = torch.empty(lib.id11b_adjoint_workspace_bytes(max(self.ngrains, 1)) // 8,
                              dtype=torch.float64, device=dev)
        # sin and cos of every peak's omega, made once: omega is fixed, so an
        # optimiser's evaluations reuse them
        self.omega_sincos = torch.empty((max(self.n, 1), 2), dtype=torch.float64, device=dev)
        check(lib.id11b_dev_omega_sincos(self.omega.data_ptr(), self.n, self.omegasign,
                                         self.omega_sincos.data_ptr(), _stream()), "omega_sincos")

    def _ptrs(self):
        return (self.det.ctypes.data, self.sc.data_ptr(), self.fc.data_ptr(),
                self.omega.data_ptr(), self.omega_sincos.data_ptr(), self.hkl.data_ptr(),
                self.offsets.data_ptr())


def _stream():
    return _torch().cuda.current_stream().cuda_stream


def _params(p):
    torch = _torch()
    p = p.detach()
    if p.dtype != torch.float64 or not p.is_cuda or p.numel() != len(PARAMS):
        raise ValueError("params: (12,) float64 CUDA tensor in the order of PARAMS")
    return p.contiguous()


class _Residuals(_torch().autograd.Function):
    """res (n,3) = UBI_G . g(params) - hkl."""

    @staticmethod
    def forward(ctx, params, ubis, peaks):
        torch = _torch()
        p = _params(params)
        u = ubis.detach().reshape(-1, 9).contiguous()
        res = torch.empty((peaks.n, 3), dtype=torch.float64, device=u.device)
        check(lib.id11b_dev_residuals(p.data_ptr(), *peaks._ptrs(), u.data_ptr(), peaks.ngrains,
                                      res.data_ptr(), None, None, _stream()), "residuals")
        ctx.peaks = peaks
        ctx.save_for_backward(p, u)
        ctx.ubi_shape = ubis.shape
        return res

    @staticmethod
    def backward(ctx, grad_res):
        torch = _torch()
        p, u = ctx.saved_tensors
        peaks = ctx.peaks
        gr = grad_res.detach().to(torch.float64).contiguous()
        gu = torch.empty_like(u)
        gp = torch.empty(len(PARAMS), dtype=torch.float64, device=u.device)
        check(lib.id11b_dev_residuals_adjoint(
            p.data_ptr(), *peaks._ptrs(), u.data_ptr(), peaks.ngrains, gr.data_ptr(),
            gu.data_ptr(), gp.data_ptr(), peaks.ws.data_ptr(), peaks.ws.numel() * 8,
            _stream()), "residuals_adjoint")
        return gp, gu.view(ctx.ubi_shape), None


class _Loss(_torch().autograd.Function):
    """0.5 * sum |res|^2, with its gradients from the same fused pass."""

    @staticmethod
    def forward(ctx, params, ubis, peaks):
        torch = _torch()
        p = _params(params)
        u = ubis.detach().reshape(-1, 9).contiguous()
        L = torch.empty((), dtype=torch.float64, device=u.device)
        gp = torch.empty(len(PARAMS), dtype=torch.float64, device=u.device)
        gu = torch.empty_like(u) if ctx.needs_input_grad[1] else None
        check(lib.id11b_dev_residual_loss(
            p.data_ptr(), *peaks._ptrs(), u.data_ptr(), peaks.ngrains, L.data_ptr(),
            gu.data_ptr() if gu is not None else None, gp.data_ptr(), None,
            peaks.ws.data_ptr(), peaks.ws.numel() * 8, _stream()), "residual_loss")
        ctx.save_for_backward(gp, gu if gu is not None else u)
        ctx.has_gu = gu is not None
        ctx.ubi_shape = ubis.shape
        return L

    @staticmethod
    def backward(ctx, grad_out):
        gp, gu = ctx.saved_tensors
        return (grad_out * gp, (grad_out * gu).view(ctx.ubi_shape) if ctx.has_gu else None,
                None)


class _ProjectedLoss(_torch().autograd.Function):
    """min over every grain's UBI of 0.5 * sum |res|^2 (variable projection):
    the loss at each grain's least-squares UBI, and its gradient with respect
    to the geometry, from one fused kernel."""

    @staticmethod
    def forward(ctx, params, peaks, ubis_out):
        torch = _torch()
        p = _params(params)
        L = torch.empty((), dtype=torch.float64, device=p.device)
        gp = torch.empty(len(PARAMS), dtype=torch.float64, device=p.device)
        check(lib.id11b_dev_residual_loss(
            p.data_ptr(), *peaks._ptrs(), None, peaks.ngrains, L.data_ptr(), None,
            gp.data_ptr(), ubis_out.data_ptr() if ubis_out is not None else None,
            peaks.ws.data_ptr(), peaks.ws.numel() * 8, _stream()), "projected_loss")
        ctx.save_for_backward(gp)
        return L

    @staticmethod
    def backward(ctx, grad_out):
        gp, = ctx.saved_tensors
        return grad_out * gp, None, None


def residuals(params, ubis, peaks):
    """Residuals (n,3) of every assigned peak, differentiable with respect to
    ``params`` -- a (12,) float64 CUDA tensor in the order of PARAMS -- and
    ``ubis`` -- (ngrains,3,3) float64 CUDA tensor."""
    return _Residuals.apply(params, ubis, peaks)


def params_tensor(geo):
    """(12,) float64 CUDA tensor of the PARAMS entries of an ImageD11-style dict."""
    torch = _torch()
    return torch.tensor([float(geo[k]) for k in PARAMS], dtype=torch.float64, device="cuda")


def gvectors(params, peaks):
    """g-vectors (n,3) of the peaks for the geometry ``params`` (no gradient)."""
    torch = _torch()
    p = _params(params)
    g = torch.empty((peaks.n, 3), dtype=torch.float64, device=p.device)
    check(lib.id11b_dev_residuals(p.data_ptr(), *peaks._ptrs(), None, peaks.ngrains, None,
                                  g.data_ptr(), None, _stream()), "gvectors")
    return g


def best_ubis(params, peaks):
    """Each grain's UBI minimising sum |UBI.g - h|^2 over its peaks for the
    g-vectors at ``params``: UBI = (sum h g^T)(sum g g^T)^-1, an FP64 3x3
    solve per grain (UBI 0 where the normal matrix B = sum g g^T is singular,
    det B <= 1e-10 trace(B)^3, as for fewer than three independent g)."""
    torch = _torch()
    p = _params(params)
    u = torch.empty((max(peaks.ngrains, 0), 3, 3), dtype=torch.float64, device=p.device)
    check(lib.id11b_dev_best_ubis(p.data_ptr(), *peaks._ptrs(), peaks.ngrains, u.data_ptr(),
                                  _stream()), "best_ubis")
    return u


def loss(params, ubis, peaks):
    """0.5 * sum of squared residuals (differentiable in params and ubis)."""
    return _Loss.apply(params, ubis, peaks)


def projected_loss(params, peaks, ubis_out=None):
    """0.5 * sum of squared residuals at every grain's least-squares UBI
    (differentiable in params); the UBIs go to ``ubis_out`` ((ngrains,3,3)
    float64 CUDA tensor) when given."""
    return _ProjectedLoss.apply(params, peaks, ubis_out)


class _BraggTheta(_torch().autograd.Function):
    @staticmethod
    def forward(ctx, ubs, peaks, wavelength):
        torch = _torch()
        b = ubs.detach().reshape(-1, 9).contiguous()
        theta = torch.empty(peaks.n, dtype=torch.float64, device=b.device)
        check(lib.id11b_dev_bragg_theta(b.data_ptr(), peaks.hkl.data_ptr(),
                                        peaks.offsets.data_ptr(), peaks.ngrains,
                                        float(wavelength), theta.data_ptr(), None, _stream()),
              "bragg_theta")
        ctx.save_for_backward(b)
        ctx.peaks, ctx.wavelength, ctx.shape = peaks, float(wavelength), ubs.shape
        return theta

    @staticmethod
    def backward(ctx, grad_theta):
        torch = _torch()
        b, = ctx.saved_tensors
        peaks = ctx.peaks
        gt = grad_theta.detach().to(torch.float64).contiguous()
        gb = torch.empty_like(b)
        check(lib.id11b_dev_bragg_theta_adjoint(b.data_ptr(), peaks.hkl.data_ptr(),
                                                peaks.offsets.data_ptr(), peaks.ngrains,
                                                ctx.wavelength, gt.data_ptr(), gb.data_ptr(),
                                                _stream()), "bragg_theta_adjoint")
        return gb.view(ctx.shape), None, None


def bragg_theta(ubs, peaks, wavelength):
    """Bragg angle theta (degrees, (n,)) of every assigned reflection computed
    from its grain's UB matrix -- ``ubs`` (ngrains,3,3) float64 CUDA tensor,
    the inverse of the UBI -- as ImageD11 src/deriv.c:38-53 computes it
    (asin(wavelength |UB h| / 2)); differentiable in ``ubs``."""
    return _BraggTheta.apply(ubs, peaks, wavelength)


def bragg_theta_jacobian(ubs, peaks, wavelength):
    """(theta (n,), dtheta/dUB (n,3,3)) per reflection, forward mode, the
    pair ImageD11 src/deriv.c:38-53 returns in tth_calc[0] and tth_calc[1:10]."""
    torch = _torch()
    b = ubs.detach().reshape(-1, 9).contiguous()
    theta = torch.empty(peaks.n, dtype=torch.float64, device=b.device)
    jac = torch.empty((peaks.n, 3, 3), dtype=torch.float64, device=b.device)
    check(lib.id11b_dev_bragg_theta(b.data_ptr(), peaks.hkl.data_ptr(), peaks.offsets.data_ptr(),
                                    peaks.ngrains, float(wavelength), theta.data_ptr(),
                                    jac.data_ptr(), _stream()), "bragg_theta")
    return theta, jac


def refine_geometry(peaks, params0, free=None, max_iter=60, history=20, max_eval=None):
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
    ``max_eval``: evaluation budget (default max_iter * 5 // 4 + 20, so that
    the line search of even one iteration can bracket its step).
    Returns (params, ubis, history of loss values); the last history entry is
    the loss at the returned params."""
    torch = _torch()
    free = [p for p in PARAMS if p != "wavelength"] if free is None else list(free)
    mask = torch.tensor([p in free for p in PARAMS], dtype=torch.float64, device="cuda")
    scale = torch.tensor([SCALES[p] for p in PARAMS], dtype=torch.float64, device="cuda")
    base = _params(params0).clone()
    x = torch.zeros(len(PARAMS), dtype=torch.float64, device="cuda", requires_grad=True)
    hist = []

    def current():
        return base + mask * scale * x

    def closure():
        opt.zero_grad()
        value = projected_loss(current(), peaks)
        value.backward()
        hist.append(float(value.detach()))
        return value

    if max_eval is None:
        max_eval = max_iter * 5 // 4 + 20
    opt = torch.optim.LBFGS([x], lr=1.0, max_iter=max_iter, max_eval=max_eval,
                            history_size=history, tolerance_grad=1e-14,
                            tolerance_change=1e-16, line_search_fn="strong_wolfe")
    opt.step(closure)
    p = current().detach()
    u = torch.empty((peaks.ngrains, 3, 3), dtype=torch.float64, device="cuda")
    with torch.no_grad():
        hist.append(float(projected_loss(p, peaks, u)))
    return p, u, hist
