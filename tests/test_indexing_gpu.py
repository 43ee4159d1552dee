"""Batched indexer.scorethem against the reference's own indexer.

tests/golden/indexer.npz (made by tests/golden/make_indexer.py) holds, for
three simulated fcc Al peak sets, the inputs and outputs of the reference's
``indexer.scorethem`` (ImageD11/indexing.py:762-874) run with the reference's
own unitcell and its own C (score, score_and_refine, score_and_assign): the
hit list, the unitcell's orientation of every hit, and the ubis, scores, ga,
hits left and the UBI handed to refine.  Here an object with the indexer's
attributes replays those orientations and runs this package's batched
scorethem, whose scoring, refinement and assignment run on the GPU.

Scores, ga and the hits left must be identical; the refined UBIs agree to
1e-12 relative (score_and_refine sums its normal equations in another order
than the reference's sequential loop)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UBI_RTOL = 1e-12


class ReplayCell:
    """unitcell.orient answering with the reference unitcell's recorded
    orientations, keyed by the two g-vectors."""

    def __init__(self, gv, hits, plain, nlist, lists):
        self.table = {}
        start = 0
        for (_, i, j), u, n in zip(hits, plain, nlist):
            i, j = int(i), int(j)
            self.table[(gv[i].tobytes(), gv[j].tobytes())] = (u, list(lists[start:start + n]))
            start += n
        self.UBI, self.UBIlist = None, []

    def orient(self, ring1, g1, ring2, g2, verbose=0, crange=-1.):
        plain, window = self.table[(np.asarray(g1).tobytes(), np.asarray(g2).tobytes())]
        if crange > 0:
            self.UBIlist = [u.copy() for u in window]
            if window:
                self.UBI = window[-1].copy()
        else:
            self.UBI = plain.copy()
            self.UBIlist = [self.UBI]


class ReplayIndexer:
    """The attributes and methods of ImageD11.indexing.indexer that
    scorethem reads, with score/getind through this package's drop-in."""

    def __init__(self, d, c):
        from imaged11_b200 import cImageD11
        k = lambda name: d["c%d_%s" % (c, name)]  # noqa: E731
        self.cim = cImageD11
        self.gv = np.ascontiguousarray(k("gv"))
        self.ra = k("ra")
        self.gvflat = np.ascontiguousarray(self.gv[self.ra > -1])
        tol, minpks, maxg, uniq, r1, r2, ctol = k("params")
        self.hkl_tol, self.minpks, self.max_grains = float(tol), int(minpks), int(maxg)
        self.uniqueness, self.ring_1, self.ring_2 = float(uniq), int(r1), int(r2)
        self.cosine_tol = float(ctol)
        self.hits = [[float(a), int(i), int(j)] for a, i, j in k("hits")]
        self.unitcell = ReplayCell(self.gv, k("hits"), k("orient_plain"), k("orient_nlist"),
                                   k("orient_list"))
        self.ga = np.zeros(len(self.gv), np.int32) - 1
        self.ubis, self.scores, self.refined = [], [], []

    def score(self, UBI, tol=None):
        return self.cim.score(UBI, self.gv, self.hkl_tol if tol is None else tol)

    def getind(self, UBI, tol=None, drlv2tmp=None, labelstmp=None):
        tol = self.hkl_tol if tol is None else tol
        drlv2 = drlv2tmp if drlv2tmp is not None else np.ones(len(self.gvflat))
        labels = labelstmp if labelstmp is not None else np.zeros(len(self.gvflat), np.int32)
        drlv2[:] = 1
        labels[:] = 0
        self.cim.score_and_assign(UBI, self.gv, tol, drlv2, labels, 1)
        return labels == 1

    def refine(self, UBI):
        self.refined.append(np.array(UBI))


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= UBI_RTOL * np.abs(b).max()


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("method", ["grid", "screen"])
def test_scorethem_matches_reference_indexer(golden, case, method, cuda):
    from imaged11_b200 import indexing
    d = golden["indexer"]
    idx = ReplayIndexer(d, case)
    want = lambda name: d["c%d_%s" % (case, name)]  # noqa: E731
    kept = indexing.scorethem(idx, method=method)
    assert kept == len(want("scores")) and kept > 0
    assert idx.scores == [int(s) for s in want("scores")]
    assert np.array_equal(idx.ga, want("ga"))
    left = np.array(idx.hits, dtype=np.float64).reshape(-1, 3)
    assert np.array_equal(left, want("hits_left"))
    assert len(idx.ubis) == len(want("ubis"))
    for u, v in zip(idx.ubis, want("ubis")):
        assert _close(u, v)
    assert len(idx.refined) == len(want("refined")) == 1
    assert _close(idx.refined[0], want("refined")[0])
