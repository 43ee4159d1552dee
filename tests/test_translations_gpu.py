"""Per-grain translation refinement (refinegrains.refinepositions objective)
against the oracle.

The objective at given translations equals the reference's gof numerator:
per grain, compute_gv at the grain's translation, one score_and_refine update
of the UBI read at tol = 1, then n * mean drlv2 of a second score_and_refine
at the updated UBI (refinegrains.refine's two calls), to the rounding of the
GPU's sin/cos (1e-9 relative).  The Gauss-Newton result reaches the simulated
translations and a cost no higher than a Nelder-Mead simplex (the reference's
method) run on the oracle's objective."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    from imaged11_b200 import synth
    geo = synth.default_geometry(distance=152300.0, tilt_x=0.004, tilt_y=-0.002,
                                 tilt_z=0.006, wedge=0.01, chi=0.02)
    ps = synth.simulate(40, "Al", gmax=1.3, seed=81, geo=geo, noise_frac=0.0,
                        translations_um=60.0, sigma_px=0.2, sigma_om=0.02)
    idx, off = ps.grain_offsets()
    p, r, dist = synth.xlylzl_params(geo)
    return ps, geo, idx, off, p, r, dist


def oracle_cost(oracle, xyz, om, ubi, t, geo):
    gv = oracle.compute_gv(xyz, om, geo["omegasign"], geo["wavelength"], geo["wedge"],
                           geo["chi"], np.asarray(t, float))
    _, _, u1 = oracle.score_and_refine(ubi, gv, 1.0)
    n, mean, _ = oracle.score_and_refine(u1, gv, 1.0)
    return n * mean, n


def test_objective_matches_oracle(scene, oracle, cuda):
    from imaged11_b200 import batch
    ps, geo, idx, off, p, r, dist = scene
    xyz = oracle.compute_xlylzl(ps.s[idx], ps.f[idx], p, r, dist)
    om = ps.omega[idx]
    rng = np.random.default_rng(82)
    t0 = rng.uniform(-80, 80, (len(off) - 1, 3))
    _, cost, npk = batch.refine_translations(xyz, om, off, ps.ubis, t0, geo["omegasign"],
                                             geo["wavelength"], geo["wedge"], geo["chi"],
                                             iters=0)
    cost, npk = cost.cpu().numpy(), npk.cpu().numpy()
    for g in range(len(off) - 1):
        a, b = off[g], off[g + 1]
        c, n = oracle_cost(oracle, xyz[a:b], om[a:b], ps.ubis[g], t0[g], geo)
        assert npk[g] == n
        assert abs(cost[g] - c) <= 1e-9 * c + 1e-15


def test_recovers_translations(scene, oracle, cuda):
    from scipy.optimize import minimize
    from imaged11_b200 import batch
    ps, geo, idx, off, p, r, dist = scene
    xyz = oracle.compute_xlylzl(ps.s[idx], ps.f[idx], p, r, dist)
    om = ps.omega[idx]
    ng = len(off) - 1
    t, cost, npk = batch.refine_translations(xyz, om, off, ps.ubis, np.zeros((ng, 3)),
                                             geo["omegasign"], geo["wavelength"], geo["wedge"],
                                             geo["chi"], iters=30)
    t, cost = t.cpu().numpy(), cost.cpu().numpy()
    err = np.abs(t - ps.translations)
    assert np.median(err) < 3.0 and err.max() < 25.0, (np.median(err), err.max())
    for g in range(0, ng, 8):     # Nelder-Mead on the oracle's objective, as the reference
        a, b = off[g], off[g + 1]
        res = minimize(lambda tt: oracle_cost(oracle, xyz[a:b], om[a:b], ps.ubis[g], tt, geo)[0],
                       np.zeros(3), method="Nelder-Mead",
                       options={"xatol": 1e-3, "fatol": 1e-12, "maxiter": 2000})
        c_gn, _ = oracle_cost(oracle, xyz[a:b], om[a:b], ps.ubis[g], t[g], geo)
        assert c_gn <= res.fun * (1 + 1e-6) + 1e-12, (g, c_gn, res.fun)
