"""Drop-in for ImageD11.refinegrains.refinegrains.refinepositions.

The reference (ImageD11/refinegrains.py:636-660) fixes the peak assignments
(assignlabels), sets the tolerance to 1.0 and then, grain by grain, runs a
Nelder-Mead simplex over t_x, t_y, t_z on gof (:517-560): the grain's
g-vectors at the trial translation (compute_gv, :366-456), two
score_and_refine calls from the UBI it was read with (refine, :459-498), and
1e6 times the mean drlv2 of the second call.

:func:`refinepositions` takes the same refinegrains object and keeps those
steps, but minimises every grain's objective at once on the GPU by damped
Gauss-Newton (csrc/translation.cu, one launch for all grains), then writes
``grains[key].translation`` as the reference does.  Supported as in the
reference's default use: triclinic lattice symmetry (no cell constraint
between the two score_and_refine calls) and omega used as observed
(``OMEGA_FLOAT`` false); other settings raise ValueError rather than
computing a different objective.
"""
import numpy as np

from . import batch


def _is_triclinic(sym):
    return getattr(sym, "__name__", None) == "triclinic"


def grain_peaks(rg, keys):
    """(xyz (n,3), omega (n,), offsets (ngrains+1,)) of the peaks assignlabels
    gave each grain in ``keys``, stacked grain by grain."""
    xyz = [np.asarray(rg.grains[k].peaks_xyz, dtype=np.float64).reshape(-1, 3) for k in keys]
    om = [np.asarray(rg.grains[k].om, dtype=np.float64).reshape(-1) for k in keys]
    off = np.zeros(len(keys) + 1, np.int64)
    off[1:] = np.cumsum([len(o) for o in om])
    if len(keys) == 0:
        return np.zeros((0, 3)), np.zeros(0), off
    return np.concatenate(xyz), np.concatenate(om), off


def refinepositions(rg, quiet=True, maxiters=100):
    """refinegrains.refinepositions with the per-grain simplex replaced by one
    batched Gauss-Newton launch: grain translations (every key of
    ``rg.grains``) minimise the reference's gof, starting from each grain's
    current translation, with the UBIs read (``rg.ubisread``) and the peak
    assignment of ``rg.assignlabels()``.  ``maxiters`` bounds the
    Gauss-Newton iterations.  Returns {key: gof} at the refined translations
    (the reference returns nothing; its gof is 1e6 * mean drlv2)."""
    if not _is_triclinic(rg.latticesymmetry):
        raise ValueError("refinepositions: only triclinic lattice symmetry is supported")
    if rg.OMEGA_FLOAT:
        raise ValueError("refinepositions: omega must be used as observed (OmFloat=False)")
    rg.assignlabels()
    keys = sorted(rg.grains.keys())
    if not keys:
        return {}
    pars = rg.parameterobj.parameters
    sign = float(pars.get("omegasign", 1.0))
    xyz, om, off = grain_peaks(rg, keys)
    ubis = np.array([rg.ubisread[k[0]] for k in keys], dtype=np.float64)
    t0 = np.array([np.asarray(rg.grains[k].translation, dtype=np.float64) for k in keys])
    tolcache = rg.tolerance
    rg.tolerance = 1.0
    try:
        t, cost, npk = batch.refine_translations(
            xyz, om, off, ubis, t0, sign, float(pars["wavelength"]), float(pars["wedge"]),
            float(pars["chi"]), tol=rg.tolerance, iters=int(maxiters))
        t, cost, npk = t.cpu().numpy(), cost.cpu().numpy(), npk.cpu().numpy()
    finally:
        rg.tolerance = tolcache
    gof = {}
    for g, k in enumerate(keys):
        tr = rg.grains[k].translation
        for i in range(3):
            tr[i] = t[g, i]
        gof[k] = 1e6 * cost[g] / npk[g] if npk[g] > 0 else 1e6
        if not quiet:
            print(k, rg.grains[k].translation, "%-8d %.6f" % (npk[g], np.sqrt(cost[g] / max(npk[g], 1))))
    # the reference leaves the last grain's translation in the parameters,
    # with the translations as the varied parameters
    rg.parameterobj.varylist = ["t_x", "t_y", "t_z"]
    for i, name in enumerate(rg.parameterobj.varylist):
        pars[name] = float(t[-1, i])
    return gof
