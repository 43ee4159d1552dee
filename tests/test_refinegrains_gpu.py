"""refinegrains.refinepositions drop-in against the reference's own run.

tests/golden/refinegrains.npz (made by tests/golden/make_refinegrains.py)
holds a scan of 10 fcc Al grains at different positions, each grain's peaks
as the reference's assignlabels left them, the UBIs read, the starting
translations, and what the reference's refinepositions (a Nelder-Mead
simplex per grain over ImageD11/refinegrains.py gof) wrote, with its gof
there.

The oracle's gof (compute_gv, then the two score_and_refine calls of
refinegrains.refine, at tolerance 1.0) reproduces the reference's gof at the
reference's translations (CPU test, 1e-12 relative).  On the GPU, the
drop-in runs on an object with the refinegrains attributes and must reach,
for every grain, a gof no higher than the simplex's (both evaluated by the
oracle), and report its own gof to 1e-9 of the oracle's."""
import numpy as np
import pytest

GEOKEYS = ("distance", "y_center", "z_center", "y_size", "z_size", "tilt_x", "tilt_y",
           "tilt_z", "o11", "o12", "o21", "o22", "omegasign", "wavelength", "wedge", "chi",
           "t_x", "t_y", "t_z")


def oracle_gof(oracle, d, g, t):
    geo = dict(zip(GEOKEYS, d["geo"]))
    a, b = d["offsets"][g], d["offsets"][g + 1]
    gv = oracle.compute_gv(d["xyz"][a:b], d["omega"][a:b], geo["omegasign"], geo["wavelength"],
                           geo["wedge"], geo["chi"], np.asarray(t, float))
    _, _, u1 = oracle.score_and_refine(d["ubis"][g], gv, 1.0)
    n, mean, _ = oracle.score_and_refine(u1, gv, 1.0)
    return 1e6 * mean


def test_oracle_gof_matches_reference(golden, oracle):
    d = golden["refinegrains"]
    for g in range(len(d["offsets"]) - 1):
        got = oracle_gof(oracle, d, g, d["t_ref"][g])
        assert abs(got - d["gof_ref"][g]) <= 1e-12 * d["gof_ref"][g]


def triclinic(cp):
    return cp


class Grain:
    def __init__(self, translation):
        self.translation = np.array(translation, dtype=np.float64)


class Parameters:
    def __init__(self, pars):
        self.parameters = dict(pars)
        self.varylist = []


class RefineGrains:
    """The refinegrains attributes refinepositions reads; assignlabels gives
    each grain the peaks the reference's assignlabels gave it."""

    def __init__(self, d):
        self.d = d
        self.latticesymmetry = triclinic
        self.OMEGA_FLOAT = False
        self.tolerance = 0.1
        self.parameterobj = Parameters(zip(GEOKEYS, d["geo"]))
        names = [int(k) for k in d["keys"]]
        self.ubisread = {n: d["ubis"][i].copy() for i, n in enumerate(names)}
        self.grains = {(n, "scan0"): Grain(d["t0"][i]) for i, n in enumerate(names)}
        self.assigned = 0

    def assignlabels(self):
        off = self.d["offsets"]
        for i, k in enumerate(sorted(self.grains)):
            self.grains[k].peaks_xyz = self.d["xyz"][off[i]:off[i + 1]]
            self.grains[k].om = self.d["omega"][off[i]:off[i + 1]]
        self.assigned += 1


@pytest.mark.gpu
def test_refinepositions_no_worse_than_reference_simplex(golden, oracle, cuda):
    from imaged11_b200 import refinegrains
    d = golden["refinegrains"]
    rg = RefineGrains(d)
    gof = refinegrains.refinepositions(rg, maxiters=100)
    assert rg.assigned == 1 and rg.tolerance == 0.1
    keys = sorted(rg.grains)
    for g, k in enumerate(keys):
        t = rg.grains[k].translation
        ours = oracle_gof(oracle, d, g, t)
        assert abs(gof[k] - ours) <= 1e-9 * ours, (g, gof[k], ours)
        assert ours <= d["gof_ref"][g] * (1 + 1e-9), (g, ours, d["gof_ref"][g])
    assert np.allclose([rg.parameterobj.parameters[n] for n in ("t_x", "t_y", "t_z")],
                       rg.grains[keys[-1]].translation)


@pytest.mark.gpu
def test_refinepositions_rejects_unsupported_settings(golden, cuda):
    from imaged11_b200 import refinegrains
    d = golden["refinegrains"]
    rg = RefineGrains(d)
    rg.OMEGA_FLOAT = True
    with pytest.raises(ValueError):
        refinegrains.refinepositions(rg)
    rg = RefineGrains(d)
    rg.latticesymmetry = lambda cp: cp
    with pytest.raises(ValueError):
        refinegrains.refinepositions(rg)
