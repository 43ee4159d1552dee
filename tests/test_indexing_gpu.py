"""Batched indexer.scorethem against the same loop scoring one hit at a time.

The indexer here is a small stand-in with the attributes and methods
ImageD11/indexing.py's indexer has (its unit cell orients a cubic cell on two
peaks of known hkl by the Busing-Levy construction).  The sequential walk
below restates the reference's scorethem loop (ImageD11/indexing.py:762-874)
with a score call per hit; the batched version must keep the same grains, in
the same order, with the same scores and peak assignments."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _unit(v):
    return v / np.sqrt((v * v).sum())


class CubicCell:
    """orient(ring1, g1, ring2, g2, verbose, crange) as ImageD11's unitcell,
    for peaks whose hkl is known (hkl_of maps a g-vector to it)."""

    def __init__(self, a, hkl_of):
        self.B = np.eye(3) / a
        self.hkl_of = hkl_of

    def _orient(self, h1, h2, g1, g2):
        h1c, h2c = self.B @ h1, self.B @ h2
        t1c, t3c = _unit(h1c), _unit(np.cross(h1c, h2c))
        t2c = _unit(np.cross(h1c, t3c))
        t1g, t3g = _unit(g1), _unit(np.cross(g1, g2))
        t2g = _unit(np.cross(g1, t3g))
        U = np.array([t1g, t2g, t3g]).T @ np.linalg.inv(np.array([t1c, t2c, t3c]).T)
        return np.linalg.inv(U @ self.B)

    def orient(self, ring1, g1, ring2, g2, verbose=0, crange=-1.):
        h1, h2 = self.hkl_of(g1), self.hkl_of(g2)
        self.UBI = self._orient(h1, h2, g1, g2)
        self.UBIlist = [self.UBI]
        if crange > 0:  # a second, worse candidate (the swapped pair)
            self.UBIlist.append(self._orient(h2, h1, g1, g2))


class Indexer:
    def __init__(self, gv, hkl, hits, tol=0.05, minpks=20):
        from imaged11_b200 import cImageD11
        self.cim = cImageD11
        self.gv = gv
        self.gvflat = np.ascontiguousarray(gv)
        lut = {tuple(g): h for g, h in zip(gv, hkl)}
        self.unitcell = CubicCell(4.05, lambda g: lut[tuple(g)])
        self.hits = list(hits)
        self.ga = np.zeros(len(gv), np.int32) - 1
        self.hkl_tol, self.minpks, self.max_grains, self.uniqueness = tol, minpks, 100, 0.5
        self.ring_1, self.ring_2, self.cosine_tol = 0, 1, 0.01
        self.ubis, self.scores = [], []
        self.refined = None

    def score(self, UBI, tol=None):
        return self.cim.score(UBI, self.gv, self.hkl_tol if tol is None else tol)

    def getind(self, UBI, tol=None, drlv2tmp=None, labelstmp=None):
        tol = self.hkl_tol if tol is None else tol
        drlv2 = drlv2tmp if drlv2tmp is not None else np.ones(len(self.gv))
        labels = labelstmp if labelstmp is not None else np.zeros(len(self.gv), np.int32)
        drlv2[:] = 1
        labels[:] = 0
        self.cim.score_and_assign(UBI, self.gv, tol, drlv2, labels, 1)
        return labels == 1

    def refine(self, UBI):
        self.refined = UBI.copy()


def sequential(idx):
    """The reference's walk, one score call per hit."""
    drlv2tmp = np.empty(len(idx.gv))
    labelstmp = np.empty(len(idx.gv), np.int32)
    ng = 0
    tol = idx.hkl_tol
    while len(idx.hits) > 0 and ng < idx.max_grains:
        _, i, j = idx.hits.pop()
        if idx.ga[i] > -1 or idx.ga[j] > -1 or i == j:
            continue
        idx.unitcell.orient(idx.ring_1, idx.gv[i], idx.ring_2, idx.gv[j], verbose=0)
        npk = idx.score(idx.unitcell.UBI, tol)
        UBI = idx.unitcell.UBI.copy()
        if npk > idx.minpks:
            idx.unitcell.orient(idx.ring_1, idx.gv[i], idx.ring_2, idx.gv[j], verbose=0,
                                crange=abs(idx.cosine_tol))
            if len(idx.unitcell.UBIlist) > 1:
                npks = [idx.score(u, tol) for u in idx.unitcell.UBIlist]
                c = int(np.argmax(npks))
                if npks[c] >= npk:
                    UBI = idx.unitcell.UBIlist[c].copy()
                    npk = npks[c]
            idx.cim.score_and_refine(UBI, idx.gvflat, tol)
            ind = idx.getind(UBI, drlv2tmp=drlv2tmp, labelstmp=labelstmp)
            ga = idx.ga[ind]
            if np.sum(np.where(ga == -1, 1, 0)) * 1.0 / ga.shape[0] > idx.uniqueness:
                idx.ga[ind] = len(idx.scores) + 1
                idx.ubis.append(UBI)
                idx.scores.append(npk)
                ng += 1
    if idx.ubis:
        idx.refine(idx.ubis[int(np.argmax(idx.scores))])


@pytest.mark.parametrize("method", ["grid", "screen"])
def test_scorethem_matches_sequential(method, cuda):
    from imaged11_b200 import indexing, synth
    ps = synth.simulate(12, "Al", gmax=1.2, seed=91, noise_frac=0.1, sigma_px=0.2,
                        sigma_om=0.02)
    lab = ps.labels
    ok = lab >= 0
    gv = np.ascontiguousarray(ps.gv)
    hkl = np.where(ok[:, None], np.nan_to_num(ps.hkl), 0.0)
    rng = np.random.default_rng(92)
    hits = []
    for _ in range(400):                        # pairs from one grain, and random pairs
        g = rng.integers(0, len(ps.ubis))
        mem = np.flatnonzero(lab == g)
        i, j = rng.choice(mem, 2, replace=True)
        if rng.random() < 0.3:
            j = rng.integers(0, len(gv))
        if not (ok[i] and ok[j]) or np.linalg.norm(np.cross(hkl[i], hkl[j])) == 0:
            continue
        hits.append((0.0, int(i), int(j)))
    a = Indexer(gv, hkl, hits)
    b = Indexer(gv, hkl, hits)
    sequential(a)
    kept = indexing.scorethem(b, method=method)
    assert kept == len(a.ubis) and kept > 0
    assert a.scores == b.scores
    assert np.array_equal(a.ga, b.ga)
    for u, v in zip(a.ubis, b.ubis):
        assert np.array_equal(u, v)
    assert np.array_equal(a.refined, b.refined)
    assert a.hits == b.hits
