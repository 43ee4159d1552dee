"""Adjoint of the assigned-peak residuals (compute_xlylzl -> compute_gv ->
UBI.g - h) with respect to the 12 geometry parameters and the UBIs.

Checked three ways: the loss against the reference's own numpy forward model,
the gradient against the reference model's central finite differences
(tests/golden/adjoint.npz), and against central finite differences of this
package's forward kernel.  Tolerance: 1e-6 relative (plus 1e-9 of the largest
component for near-zero entries)."""
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
    return float(L), p.grad.cpu().numpy(), u.grad.cpu().numpy()


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
