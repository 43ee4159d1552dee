"""Adjoint of the assigned-peak residuals (compute_xlylzl -> compute_gv ->
UBI.g - h) with respect to the 12 geometry parameters and the UBIs.

Checked against the reference in four ways: the loss against the
reference's own numpy forward model, the gradient against the reference
model's central finite differences (tests/golden/adjoint.npz), the
translation Jacobian dg/dt against the reference's hand-derived
fittrans2.d_XSXB_to_gv and the Bragg angle derivative dtheta/dUB against its
src/deriv.c g_to_k (tests/golden/derivatives.npz); and against central
finite differences of this package's forward kernel.  Tolerance for finite
differences: 1e-6 relative (plus 1e-9 of the largest component for near-zero
entries); for the hand-derived derivatives 1e-9 and 1e-12."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-6


def _peaks(d):
    from imaged11_b200 import adjoint
    ys, zs, osg, o11, o12, o21, o22 = d["adj_const"]
    geo = dict(y_size=ys, z_size=zs, omegasign=osg, o11=o11, o12=o12, o21=o21, o22=o22)
    return adjoint.PeakTable(d["adj_s"], d["adj_f"], d["adj_omega"], d["adj_hkl"],
                             d["adj_offsets"], geo)


def _grad(params, ubis, peaks):
    from imaged11_b200 import adjoint
    p = params.clone().requires_grad_(True)
    u = ubis.clone().requires_grad_(True)
    L = adjoint.loss(p, u, peaks)
    L.backward()
    return float(L.detach()), p.grad.cpu().numpy(), u.grad.cpu().numpy()


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= GRAD_RTOL * np.abs(b) + 1e-9 * np.abs(b).max())


def test_loss_and_gradient_match_reference(golden, cuda):
    import torch
    d = golden["adjoint"]
    peaks = _peaks(d)
    params = torch.tensor(d["adj_params"], dtype=torch.float64, device=cuda)
    ubis = torch.tensor(d["adj_ubis"], dtype=torch.float64, device=cuda)
    L, gp, gu = _grad(params, ubis, peaks)
    assert abs(L - float(d["adj_loss"])) <= 1e-9 * float(d["adj_loss"])
    assert _close(gp, d["adj_grad_fd"]), np.abs(gp - d["adj_grad_fd"]) / np.abs(d["adj_grad_fd"])
    for (G, i, j), ref in zip(d["adj_grad_ubi_idx"], d["adj_grad_ubi_fd"]):
        assert abs(gu[G, i, j] - ref) <= GRAD_RTOL * abs(ref) + 1e-9


def test_gradient_matches_own_central_differences(golden, cuda):
    import torch
    from imaged11_b200 import adjoint
    d = golden["adjoint"]
    peaks = _peaks(d)
    params = torch.tensor(d["adj_params"], dtype=torch.float64, device=cuda)
    ubis = torch.tensor(d["adj_ubis"], dtype=torch.float64, device=cuda)
    _, gp, gu = _grad(params, ubis, peaks)
    fd = []
    for i, name in enumerate(adjoint.PARAMS):
        h = 1e-6 * adjoint.SCALES[name]
        e = torch.zeros_like(params)
        e[i] = h
        lp = float(adjoint.loss(params + e, ubis, peaks))
        lm = float(adjoint.loss(params - e, ubis, peaks))
        fd.append((lp - lm) / (2 * h))
    assert _close(gp, fd), np.abs(gp - np.array(fd)) / np.abs(fd)
    # a full UBI of one grain
    G = 2
    for i in range(3):
        for j in range(3):
            e = torch.zeros_like(ubis)
            e[G, i, j] = 1e-7
            num = (float(adjoint.loss(params, ubis + e, peaks)) -
                   float(adjoint.loss(params, ubis - e, peaks))) / 2e-7
            assert abs(gu[G, i, j] - num) <= GRAD_RTOL * abs(num) + 1e-9


def test_residuals_match_compute_gv(golden, cuda):
    """The adjoint's forward g equals the drop-in compute_xlylzl + compute_gv."""
    import torch
    from imaged11_b200 import adjoint, synth
    from imaged11_b200 import cImageD11 as cim
    d = golden["adjoint"]
    peaks = _peaks(d)
    params = torch.tensor(d["adj_params"], dtype=torch.float64, device=cuda)
    g = adjoint.gvectors(params, peaks).cpu().numpy()
    geo = dict(zip(adjoint.PARAMS, d["adj_params"]))
    ys, zs, osg, o11, o12, o21, o22 = d["adj_const"]
    geo.update(y_size=ys, z_size=zs, omegasign=osg, o11=o11, o12=o12, o21=o21, o22=o22)
    p, r, dist = synth.xlylzl_params(geo)
    xyz = np.empty((len(d["adj_s"]), 3))
    cim.compute_xlylzl(d["adj_s"], d["adj_f"], p, r.ravel(), dist, xyz)
    ref = np.empty_like(xyz)
    cim.compute_gv(xyz, d["adj_omega"], osg, geo["wavelength"], geo["wedge"], geo["chi"],
                   [geo["t_x"], geo["t_y"], geo["t_z"]], ref)
    assert np.abs(g - ref).max() <= 1e-12 * np.abs(ref).max()


def test_joint_refinement_recovers_geometry(cuda):
    """cfg3-like: simulated with tilts, wedge, chi, translation and offset
    centres; refined from the nominal zero-tilt geometry with the UBIs free.

    With every grain at one common translation and free orientations, two
    directions are unidentifiable from the peaks: t_z moves the spots exactly
    as a z_center shift does (the omega axis is z), and tilt_x trades against
    chi (both rotate about the beam).  The test checks the identifiable
    parameters and those two invariant combinations."""
    import math
    from imaged11_b200 import adjoint, synth
    truth = synth.default_geometry(distance=152300., y_center=1024 + 3.7,
                                   z_center=1024 - 2.1, tilt_x=0.004, tilt_y=-0.002,
                                   tilt_z=0.006, wedge=0.01, chi=0.02, t_x=5., t_y=-3., t_z=2.)
    ps = synth.simulate(40, "Al", gmax=1.3, seed=3, geo=truth, sigma_px=0.0, sigma_om=0.0,
                        noise_frac=0.0, translation=(5., -3., 2.))
    idx, off = ps.grain_offsets()
    peaks = adjoint.PeakTable(ps.s[idx], ps.f[idx], ps.omega[idx], ps.hkl[idx], off, truth)
    nominal = dict(truth, distance=150000., y_center=1024., z_center=1024., tilt_x=0.,
                   tilt_y=0., tilt_z=0., wedge=0., chi=0., t_x=0., t_y=0., t_z=0.)
    p, ubis, hist = adjoint.refine_geometry(peaks, adjoint.params_tensor(nominal), max_iter=200)
    assert hist[-1] < 1e-9 * hist[0]
    got = dict(zip(adjoint.PARAMS, p.cpu().numpy()))
    diff = {k: got[k] - truth[k] for k in adjoint.PARAMS}
    assert abs(diff["distance"]) < 0.05
    assert abs(diff["y_center"]) < 1e-3
    assert abs(diff["tilt_y"]) < 1e-7 and abs(diff["tilt_z"]) < 1e-7
    assert abs(diff["wedge"]) < 1e-6
    assert abs(diff["t_x"]) < 0.02 and abs(diff["t_y"]) < 0.02
    # the invariant combinations along the two degenerate directions
    assert abs(diff["z_center"] * truth["z_size"] + diff["t_z"]) < 0.01
    assert abs(diff["tilt_x"] - math.radians(diff["chi"])) < 1e-6


def _der_peaks(d):
    from imaged11_b200 import adjoint
    ys, zs, osg, o11, o12, o21, o22 = d["der_const"]
    geo = dict(y_size=ys, z_size=zs, omegasign=osg, o11=o11, o12=o12, o21=o21, o22=o22)
    return adjoint.PeakTable(d["der_s"], d["der_f"], d["der_omega"], d["der_hkl"],
                             d["der_offsets"], geo)


def test_translation_jacobian_matches_fittrans2(golden, cuda):
    """dg/dt from the adjoint (one reverse pass per g component, UBI = I and
    hkl = 0 so that res = g) against the reference's hand-derived
    d_XSXB_to_gv (ImageD11/sandbox/fittrans2.py:39-77), with wedge 0.3 and
    chi -0.2 degrees: g to 1e-12, dg/dt to 1e-9 relative."""
    import torch
    from imaged11_b200 import adjoint
    d = golden["derivatives"]
    peaks = _der_peaks(d)
    peaks.hkl.zero_()
    params = torch.tensor(d["der_params"], dtype=torch.float64, device=cuda)
    eye = torch.eye(3, dtype=torch.float64, device=cuda).expand(peaks.ngrains, 3, 3).contiguous()
    g = adjoint.gvectors(params, peaks).cpu().numpy()
    assert np.abs(g - d["der_g"]).max() <= 1e-12 * np.abs(d["der_g"]).max()
    sel = np.arange(0, peaks.n, max(1, peaks.n // 24))
    p = params.clone().requires_grad_(True)
    res = adjoint.residuals(p, eye, peaks)
    assert np.abs(res.detach().cpu().numpy() - d["der_g"]).max() <= 1e-12
    for k in sel:
        for i in range(3):
            gp, = torch.autograd.grad(res[k, i], p, retain_graph=True)
            dgdt = gp[9:12].cpu().numpy()
            ref = d["der_dgdt"][k, i]
            assert np.all(np.abs(dgdt - ref) <= 1e-9 * np.abs(ref).max() + 1e-15), (k, i)


def test_bragg_theta_matches_deriv_c(golden, cuda):
    """theta and dtheta/dUB against the reference's src/deriv.c:38-53
    (g_to_k), and the reverse pass against the forward Jacobian."""
    import torch
    from imaged11_b200 import adjoint
    d = golden["derivatives"]
    peaks = _der_peaks(d)
    ubs = torch.tensor(d["der_ubs"], dtype=torch.float64, device=cuda)
    lam = float(d["der_params"][6])
    th, jac = adjoint.bragg_theta_jacobian(ubs, peaks, lam)
    assert np.abs(th.cpu().numpy() - d["der_theta"]).max() <= 1e-12 * np.abs(d["der_theta"]).max()
    J = jac.cpu().numpy().reshape(-1, 9)
    assert np.all(np.abs(J - d["der_dtheta"]) <= 1e-12 * np.abs(d["der_dtheta"]).max())
    u = ubs.clone().requires_grad_(True)
    w = torch.linspace(-1, 1, peaks.n, dtype=torch.float64, device=cuda)
    (adjoint.bragg_theta(u, peaks, lam) * w).sum().backward()
    off = d["der_offsets"]
    want = np.stack([(w.cpu().numpy()[off[G]:off[G + 1], None] * J[off[G]:off[G + 1]]).sum(0)
                     for G in range(len(off) - 1)])
    assert np.allclose(u.grad.cpu().numpy().reshape(-1, 9), want, rtol=1e-12, atol=1e-12)


def test_fused_loss_equals_residual_autograd(golden, cuda):
    """The fused loss + gradient pass against 0.5 * sum(res^2) differentiated
    through the residual adjoint."""
    import torch
    from imaged11_b200 import adjoint
    d = golden["adjoint"]
    peaks = _peaks(d)
    params = torch.tensor(d["adj_params"], dtype=torch.float64, device=cuda)
    ubis = torch.tensor(d["adj_ubis"], dtype=torch.float64, device=cuda)
    p1, u1 = params.clone().requires_grad_(True), ubis.clone().requires_grad_(True)
    L1 = adjoint.loss(p1, u1, peaks)
    L1.backward()
    p2, u2 = params.clone().requires_grad_(True), ubis.clone().requires_grad_(True)
    r = adjoint.residuals(p2, u2, peaks)
    L2 = 0.5 * (r * r).sum()
    L2.backward()
    assert abs(float(L1.detach()) - float(L2.detach())) <= 1e-12 * float(L2.detach())
    assert _close(p1.grad.cpu().numpy(), p2.grad.cpu().numpy())
    assert np.allclose(u1.grad.cpu().numpy(), u2.grad.cpu().numpy(), rtol=1e-10, atol=1e-12)


def test_best_ubis_and_projected_gradient(golden, cuda):
    """Per-grain least-squares UBIs against numpy's lstsq on the same g, the
    projected loss against loss() at those UBIs, and its geometry gradient
    against central differences of the projected loss (1e-6)."""
    import torch
    from imaged11_b200 import adjoint
    d = golden["adjoint"]
    peaks = _peaks(d)
    params = torch.tensor(d["adj_params"], dtype=torch.float64, device=cuda)
    g = adjoint.gvectors(params, peaks).cpu().numpy()
    u = adjoint.best_ubis(params, peaks)
    off = d["adj_offsets"]
    for G in range(len(off) - 1):
        gg, hh = g[off[G]:off[G + 1]], d["adj_hkl"][off[G]:off[G + 1]]
        X, *_ = np.linalg.lstsq(gg, hh, rcond=None)
        assert np.allclose(u[G].cpu().numpy(), X.T, rtol=1e-10, atol=1e-12)
    uo = torch.empty_like(u)
    p = params.clone().requires_grad_(True)
    Lp = adjoint.projected_loss(p, peaks, uo)
    Lp.backward()
    assert np.array_equal(uo.cpu().numpy(), u.cpu().numpy())
    assert abs(float(Lp) - float(adjoint.loss(params, u, peaks))) <= 1e-12 * float(Lp)
    # wavelength is a flat direction of the projected loss (a common scale of
    # g and of every UBI leaves it unchanged): its derivative vanishes, and a
    # central difference there is rounding noise
    gp = p.grad.cpu().numpy()
    iw = adjoint.PARAMS.index("wavelength")
    assert abs(gp[iw]) * float(params[iw]) <= 1e-9 * float(Lp)
    fd = []
    for i, name in enumerate(adjoint.PARAMS):
        if i == iw:
            continue
        h = 1e-6 * adjoint.SCALES[name]
        e = torch.zeros_like(params)
        e[i] = h
        fd.append((float(adjoint.projected_loss(params + e, peaks)) -
                   float(adjoint.projected_loss(params - e, peaks))) / (2 * h))
    got = np.delete(gp, iw)
    assert _close(got, fd), np.abs(got - fd) / np.abs(fd)


def test_singular_grain_gets_zero_ubi(cuda):
    """A grain with two peaks has a singular normal matrix: UBI 0, finite loss
    and gradient."""
    import torch
    from imaged11_b200 import adjoint, synth
    geo = synth.default_geometry()
    ps = synth.simulate(2, "Al", gmax=1.0, seed=4, geo=geo, noise_frac=0.0)
    idx, off = ps.grain_offsets()
    off = np.concatenate([off, [off[-1] + 2]])
    idx = np.concatenate([idx, idx[:2]])
    peaks = adjoint.PeakTable(ps.s[idx], ps.f[idx], ps.omega[idx], ps.hkl[idx], off, geo)
    params = adjoint.params_tensor(geo)
    u = adjoint.best_ubis(params, peaks).cpu().numpy()
    assert np.all(u[-1] == 0) and np.all(np.abs(u[:-1]).max((1, 2)) > 0)
    p = params.clone().requires_grad_(True)
    L = adjoint.projected_loss(p, peaks)
    L.backward()
    assert np.isfinite(float(L)) and np.all(np.isfinite(p.grad.cpu().numpy()))
