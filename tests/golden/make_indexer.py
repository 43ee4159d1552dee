"""Generate tests/golden/indexer.npz from the REFERENCE's own indexer.

Run where an ImageD11 checkout exists, naming its root (argument or the
IMAGED11_REF environment variable), after ``make -C oracle REF=<root>``:

    python tests/golden/make_indexer.py /path/to/ImageD11

ImageD11.indexing and ImageD11.unitcell are imported from the checkout with
stand-ins for what they import but these cases do not use (xfab, h5py,
fabio), and with ImageD11.cImageD11 served by the reference's own C compiled
unmodified into oracle/_ref/libimaged11_ref.so: score, score_and_refine,
score_and_assign (src/closest.c), closest (src/closest.c:188-206),
quickorient (src/cdiffraction.c:293-328) and compute_gv
(src/cdiffraction.c:112-168), called with f2py's conventions.

For each case an ``indexer`` is built on a simulated fcc Al peak set, rings
are assigned (assigntorings), hits are found (find), and ``scorethem``
(ImageD11/indexing.py:762-874) runs.  The fixture holds the inputs (g-vectors,
parameters, ring assignments, the hit list), the reference unitcell's
orientation of every hit (plain, and the list within the cosine window), and
the outputs: ubis, scores, ga, the hits left and the UBI passed to refine.
The GPU test replays the recorded orientations through this package's
batched scorethem and compares.  Only the .npz file is read by the tests.
"""
import ctypes
import logging
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)

from imaged11_b200 import synth  # noqa: E402

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _cd(a):
    return a.ctypes.data_as(_D)


def reference_cimaged11(so):
    """A cImageD11 module whose functions call the reference's C."""
    L = ctypes.CDLL(so)
    L.score.argtypes = [_D, _D, ctypes.c_double, ctypes.c_int]
    L.score.restype = ctypes.c_int
    L.score_and_refine.argtypes = [_D, _D, ctypes.c_double, _I, _D, ctypes.c_int]
    L.score_and_assign.argtypes = [_D, _D, ctypes.c_double, _D, _I, ctypes.c_int,
                                   ctypes.c_int]
    L.score_and_assign.restype = ctypes.c_int
    L.closest.argtypes = [_D, _D, _I, _D, ctypes.c_int, ctypes.c_int]
    L.quickorient.argtypes = [_D, _D]
    L.compute_gv.argtypes = [_D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, _D, _D, ctypes.c_int]
    m = types.ModuleType("ImageD11.cImageD11")

    def f64(a):
        a = np.asarray(a)
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return a

    def score(ubi, gv, tol):
        g = np.ascontiguousarray(gv, dtype=np.float64)
        return int(L.score(_cd(np.ascontiguousarray(ubi, dtype=np.float64)), _cd(g),
                           float(tol), len(g)))

    def score_and_refine(ubi, gv, tol):
        u = f64(ubi)
        g = np.ascontiguousarray(gv, dtype=np.float64)
        n, s = ctypes.c_int(0), ctypes.c_double(0.)
        L.score_and_refine(_cd(u), _cd(g), float(tol), ctypes.byref(n), ctypes.byref(s), len(g))
        return n.value, s.value

    def score_and_assign(ubi, gv, tol, drlv2, labels, label):
        g = np.ascontiguousarray(gv, dtype=np.float64)
        d = f64(drlv2)
        assert labels.dtype == np.int32 and labels.flags.c_contiguous
        return int(L.score_and_assign(_cd(np.ascontiguousarray(ubi, dtype=np.float64)), _cd(g),
                                      float(tol), _cd(d), labels.ctypes.data_as(_I), int(label),
                                      len(g)))

    def closest(x, v):
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        i, b = ctypes.c_int(0), ctypes.c_double(0.)
        L.closest(_cd(x), _cd(v), ctypes.byref(i), ctypes.byref(b), len(x), len(v))
        return i.value, b.value

    def quickorient(ubi, bt):
        L.quickorient(_cd(f64(ubi)), _cd(np.ascontiguousarray(bt, dtype=np.float64)))

    def compute_gv(xyz, omega, omegasign, wvln, wedge, chi, t, gv):
        x = np.ascontiguousarray(xyz, dtype=np.float64)
        o = np.ascontiguousarray(omega, dtype=np.float64)
        tt = np.ascontiguousarray(t, dtype=np.float64)
        out = f64(gv)
        assert out.shape == x.shape
        L.compute_gv(_cd(x), _cd(o), float(omegasign), float(wvln), float(wedge), float(chi),
                     _cd(tt), _cd(out), len(o))

    m.score, m.score_and_refine, m.score_and_assign = score, score_and_refine, score_and_assign
    m.closest, m.quickorient, m.compute_gv = closest, quickorient, compute_gv
    return m


def import_reference_indexing(ref_root, so):
    for name in ("fabio", "h5py"):
        sys.modules.setdefault(name, types.ModuleType(name))
    xfab = types.ModuleType("xfab")
    xfab.__path__ = []
    tools = types.ModuleType("xfab.tools")
    for f in ("ubi_to_u", "u_to_rod", "ubi_to_rod", "genhkl_all", "form_b_mat", "ubi_to_cell"):
        setattr(tools, f, None)
    xlog = types.ModuleType("xfab.xfab_logging")
    xlog.get_module_level_logger = logging.getLogger
    xfab.tools, xfab.xfab_logging = tools, xlog
    sys.modules.update({"xfab": xfab, "xfab.tools": tools, "xfab.xfab_logging": xlog})
    pkg = types.ModuleType("ImageD11")
    pkg.__path__ = [os.path.join(ref_root, "ImageD11")]
    sys.modules["ImageD11"] = pkg
    cim = reference_cimaged11(so)
    sys.modules["ImageD11.cImageD11"] = cim
    pkg.cImageD11 = cim
    import importlib
    uc = importlib.import_module("ImageD11.unitcell")
    ix = importlib.import_module("ImageD11.indexing")
    return uc, ix


CASES = [
    # (grains, seed, cosine_tol, max_grains, minpks)
    (16, 31, 0.002, 100, 30),     # closest cosine per ring-1 peak
    (16, 32, -0.002, 100, 30),    # every pair within the window (negative tol)
    (16, 33, -0.002, 5, 30),      # stops at max_grains, hits left over
]


def run_case(uc, ix, ngrains, seed, cosine_tol, max_grains, minpks):
    ps = synth.simulate(ngrains, "Al", gmax=1.3, seed=seed, noise_frac=0.1, sigma_px=0.2,
                        sigma_om=0.02)
    gv = np.ascontiguousarray(ps.gv)
    cell = uc.unitcell([4.05, 4.05, 4.05, 90., 90., 90.], "F")
    idx = ix.indexer(unitcell=cell, gv=gv, wavelength=ps.geo["wavelength"], hkl_tol=0.05,
                     minpks=minpks, ring_1=0, ring_2=1, ds_tol=0.01, cosine_tol=cosine_tol,
                     max_grains=max_grains, uniqueness=0.5)
    idx.assigntorings()
    idx.find()
    hits = [(float(d), int(i), int(j)) for d, i, j in idx.hits]
    assert len(hits) > 0
    # the reference unitcell's orientation of every hit
    plain, nlist, lists = [], [], []
    for _, i, j in hits:
        if i == j:
            plain.append(np.zeros((3, 3)))
            nlist.append(0)
            continue
        cell.orient(idx.ring_1, gv[i], idx.ring_2, gv[j], verbose=0)
        plain.append(np.array(cell.UBI, dtype=np.float64))
        cell.orient(idx.ring_1, gv[i], idx.ring_2, gv[j], verbose=0,
                    crange=abs(idx.cosine_tol))
        nlist.append(len(cell.UBIlist))
        lists.extend(np.array(u, dtype=np.float64) for u in cell.UBIlist)
    refined = []
    ref_refine = idx.refine

    def record_refine(UBI):
        refined.append(np.array(UBI, dtype=np.float64))
        return ref_refine(UBI)

    idx.refine = record_refine
    ra = idx.ra.copy()
    idx.scorethem()
    left = np.array([(d, i, j) for d, i, j in idx.hits], dtype=np.float64).reshape(-1, 3)
    print("case: %d peaks, %d hits, %d grains kept, %d hits left" %
          (len(gv), len(hits), len(idx.ubis), len(left)))
    return dict(gv=gv, ra=ra, hits=np.array(hits, dtype=np.float64),
                params=np.array([idx.hkl_tol, idx.minpks, idx.max_grains, idx.uniqueness,
                                 idx.ring_1, idx.ring_2, idx.cosine_tol]),
                orient_plain=np.array(plain), orient_nlist=np.array(nlist, dtype=np.int64),
                orient_list=np.array(lists).reshape(-1, 3, 3),
                ubis=np.array(idx.ubis, dtype=np.float64).reshape(-1, 3, 3),
                scores=np.array(idx.scores, dtype=np.int64), ga=idx.ga.copy(),
                hits_left=left, refined=np.array(refined).reshape(-1, 3, 3))


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMAGED11_REF")
    if not ref_root:
        sys.exit("usage: make_indexer.py /path/to/ImageD11 (or set IMAGED11_REF)")
    so = os.path.join(REPO, "oracle", "_ref", "libimaged11_ref.so")
    if not os.path.exists(so):
        sys.exit("build the reference's C first: make -C oracle REF=" + ref_root)
    logging.disable(logging.CRITICAL)
    uc, ix = import_reference_indexing(ref_root, so)
    out = {}
    for c, args in enumerate(CASES):
        for k, v in run_case(uc, ix, *args).items():
            out["c%d_%s" % (c, k)] = v
    path = os.path.join(HERE, "indexer.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
