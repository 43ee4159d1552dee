"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Run where an ImageD11 checkout exists, naming its root (argument or the
IMAGED11_REF environment variable):

    make -C oracle REF=/path/to/ImageD11   # builds oracle/_ref/libimaged11_ref.so
                                           # from the reference's own C sources
    python tests/golden/make_golden.py /path/to/ImageD11

Outputs come from two reference implementations:

* the reference's compiled C (unmodified sources, via oracle/_ref) for every
  hot-path function: compute_gv, compute_geometry, compute_xlylzl, score,
  score_and_refine, refine_assigned, score_and_assign;
* the reference's numpy module ImageD11/transform.py (compute_tth_eta_from_xyz
  + compute_g_vectors, compute_xyz_lab, detector_rotation_matrix), imported
  with stub ``fabio``/``cImageD11`` modules because only its numpy functions
  are used.

The derivatives fixture holds the reference's own hand-derived derivatives:
dg/dt of ImageD11/sandbox/fittrans2.py (d_XSXB_to_gv, its function
definitions run from the file) and theta, dtheta/dUB of src/deriv.c (g_to_k,
compiled by ``make -C oracle deriv`` with its main renamed).

The adjoint fixture holds the reference forward model's loss and its central
finite-difference gradients (compute_xyz_lab -> compute_tth_eta_from_xyz ->
compute_g_vectors -> UBI.g - h) with respect to the 12 geometry parameters
and a few UBI elements.

Inputs: the cases of the reference's own test/test_cImageD11.py (7 wedge /
chi / translation / omegasign sets on 203 points; 8 detector flips x 27 tilt
triples), seeded synthetic peak sets from imaged11_b200.synth, and adversarial
scoring cases (fractional parts at 0.5 +- k ulp, drlv2 at tol^2 +- ulp,
singular normal matrices, non-finite and huge g-vectors).

The fixtures are small .npz files committed beside this script; the tests
read only the .npz files, never the reference.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)

from oracle.oracle import Reference  # noqa: E402
from imaged11_b200 import synth  # noqa: E402


def import_reference_transform(ref_root):
    """ImageD11.transform with stubbed heavy imports (fabio, cImageD11)."""
    sys.modules.setdefault("fabio", types.ModuleType("fabio"))
    pkg = types.ModuleType("ImageD11")
    pkg.__path__ = [os.path.join(ref_root, "ImageD11")]
    sys.modules["ImageD11"] = pkg
    cim = types.ModuleType("ImageD11.cImageD11")
    sys.modules["ImageD11.cImageD11"] = cim
    pkg.cImageD11 = cim
    import importlib
    gvg = importlib.import_module("ImageD11.gv_general")
    pkg.gv_general = gvg
    return importlib.import_module("ImageD11.transform")


def cases_compute_gv(ref, tr):
    """test/test_cImageD11.py:14-128 inputs, plus a seeded random set."""
    N = 203
    XLYLZL = np.array([np.linspace(0, 2000, N), np.linspace(10, 2010, N), np.ones(N)])
    omega = np.linspace(-180, 180, N)
    params = [  # wedge, chi, omegasign, wvln, t_x, t_y, t_z
        (5., 10., 1.0, 0.125, 20., 30., 40.),
        (5., 0., 1.0, 0.125, 20., 30., 40.),
        (0., 5., 1.0, 0.125, 20., 30., 40.),
        (5., 10., -1.0, 0.125, 200., 300., 40.),
        (5., 0., 1.0, 0.125, 200., 300., -400.),
        (0., 0., 1.0, 0.125, 0., 0., 0.),
        (0., 0., 1.0, 0.125, 200., 300., 400.),
    ]
    out = {}
    for i, (w, c, osg, wl, tx, ty, tz) in enumerate(params):
        t = np.array([tx, ty, tz])
        gv = ref.compute_gv(XLYLZL.T.copy(), omega, osg, wl, w, c, t)
        tth, eta = tr.compute_tth_eta_from_xyz(XLYLZL, omega * osg, t_x=tx, t_y=ty, t_z=tz,
                                               wedge=w, chi=c)
        gnp = tr.compute_g_vectors(tth, eta, omega * osg, wl, wedge=w, chi=c).T
        geom = ref.compute_geometry(XLYLZL.T.copy(), omega, osg, wl, w, c, t)
        out["gv%d_params" % i] = np.array([osg, wl, w, c, tx, ty, tz])
        out["gv%d_out" % i] = gv
        out["gv%d_numpy" % i] = gnp
        out["gv%d_geometry" % i] = geom
    out["gv_xlylzl"] = XLYLZL.T.copy()
    out["gv_omega"] = omega
    out["gv_ncases"] = np.array(len(params))
    # seeded random lab positions on a realistic detector, nonzero wedge/chi/t
    rng = np.random.default_rng(20240611)
    n = 4096
    x = np.stack([rng.uniform(1.4e5, 1.6e5, n), rng.uniform(-8e4, 8e4, n),
                  rng.uniform(-8e4, 8e4, n)], 1)
    om = rng.uniform(-180, 360, n)
    t = np.array([5., -3., 2.])
    out["rand_xlylzl"] = x
    out["rand_omega"] = om
    out["rand_params"] = np.array([-1.0, 0.2846, 0.01, 0.02, 5., -3., 2.])
    out["rand_gv"] = ref.compute_gv(x, om, -1.0, 0.2846, 0.01, 0.02, t)
    out["rand_geometry"] = ref.compute_geometry(x, om, -1.0, 0.2846, 0.01, 0.02, t)
    return out


def cases_xlylzl(ref, tr):
    """test/test_cImageD11.py:132-190: 8 flips x 27 tilts."""
    rng = np.random.default_rng(7)
    npk = 64
    sc = rng.random(npk) * 2048
    fc = rng.random(npk) * 2048
    pars = dict(z_center=980., y_center=1010., z_size=48., y_size=49., distance=100100.)
    p = np.array([pars["z_center"], pars["y_center"], pars["z_size"], pars["y_size"]])
    dist = np.array([pars["distance"], 0., 0.])
    tilts = [(x, y, z) for x in (-0.5, 0., 0.24) for y in (-0.5, 0., 0.24)
             for z in (-0.5, 0., 0.24)]
    flips = [[1, 0, 0, 1], [-1, 0, 0, 1], [-1, 0, 0, -1], [1, 0, 0, -1],
             [0, 1, 1, 0], [0, -1, 1, 0], [0, -1, -1, 0], [0, 1, -1, 0]]
    R, OUT, NP = [], [], []
    for o11, o12, o21, o22 in flips:
        for tx, ty, tz in tilts:
            kw = dict(pars, tilt_x=tx, tilt_y=ty, tilt_z=tz, o11=o11, o12=o12, o21=o21, o22=o22)
            dmat = tr.detector_rotation_matrix(tx, ty, tz)
            fmat = np.array([[1, 0, 0], [0, o22, o21], [0, o12, o11]], float)
            r = np.dot(dmat, fmat)
            R.append(r.ravel())
            OUT.append(ref.compute_xlylzl(sc, fc, p, r.ravel(), dist))
            NP.append(tr.compute_xyz_lab((sc, fc), **kw).T)
    return dict(xl_s=sc, xl_f=fc, xl_p=p, xl_dist=dist, xl_r=np.array(R), xl_out=np.array(OUT),
                xl_numpy=np.array(NP))


def adversarial_gv(ubi, rng):
    """g-vectors that put h = UBI.g exactly on rounding / tolerance edges."""
    ub = np.linalg.inv(ubi)
    hs = []
    base = rng.integers(-6, 7, size=(64, 3)).astype(float)
    # fractional parts at +-0.5 and a few ulps either side
    for k in (-3, -1, 0, 1, 3):
        h = base.copy()
        h[:, 0] = np.floor(h[:, 0]) + 0.5
        h[:, 0] = h[:, 0] + k * np.spacing(h[:, 0])
        hs.append(h)
    # drlv2 == tol^2 (+- ulp) on one component for tol in (0.02, 0.05, 0.1)
    for tol in (0.02, 0.05, 0.1):
        for k in (-2, -1, 0, 1, 2):
            h = base.copy()
            h[:, 1] = h[:, 1] + tol + k * np.spacing(tol)
            hs.append(h)
    h = np.concatenate(hs)
    g = h @ ub.T
    # back-solve so that UBI.g lands as close as possible in FP64
    return g


def cases_scoring(ref):
    out = {}
    # realistic scene: FCC Al, 40 grains, noise peaks, cfg0-like geometry
    ps = synth.simulate(40, "Al", gmax=1.2, seed=11, noise_frac=0.10)
    gv = ps.gv
    rng = np.random.default_rng(12)
    ubis = np.concatenate([synth.perturb_ubis(ps.ubis[:20], 0.1, 0.001, rng),
                           synth.trial_ubis(ps.ubis, 12, 0.0, 0.0, rng),
                           ps.ubis[20:24]])
    tols = np.array([0.02, 0.05, 0.1, 0.25])
    out["sc_gv"] = gv
    out["sc_ubis"] = ubis
    out["sc_tols"] = tols
    out["sc_counts"] = np.array([[ref.score(u, gv, t) for t in tols] for u in ubis], np.int32)
    n, d, u2 = [], [], []
    for u in ubis:
        for t in tols:
            a, b, c = ref.score_and_refine(u, gv, t)
            n.append(a); d.append(b); u2.append(c)
    out["sar_n"] = np.array(n, np.int32).reshape(len(ubis), len(tols))
    out["sar_drlv2"] = np.array(d).reshape(len(ubis), len(tols))
    out["sar_ubi"] = np.array(u2).reshape(len(ubis), len(tols), 3, 3)
    # three iterations of score_and_refine per UBI at tol 0.05 (cfg0 procedure)
    it = []
    for u in ubis[:20]:
        uu = u.copy()
        for _ in range(3):
            _, _, uu = ref.score_and_refine(uu, gv, 0.05)
        it.append(uu)
    out["sar3_ubi"] = np.array(it)
    # refine_assigned over the true labels
    labels = ps.labels.astype(np.int32)
    ra_n, ra_d, ra_u = [], [], []
    for gi in range(8):
        a, b, c = ref.refine_assigned(ubis[gi], gv, labels, gi)
        ra_n.append(a); ra_d.append(b); ra_u.append(c)
    out["ra_labels"] = labels
    out["ra_n"] = np.array(ra_n, np.int32)
    out["ra_drlv2"] = np.array(ra_d)
    out["ra_ubi"] = np.array(ra_u)
    # score_and_assign, sequentially over the first 24 UBIs (as refinegrains.assignlabels)
    drl = np.full(len(gv), 2.0)
    lab = np.full(len(gv), -1, np.int32)
    sa_n = []
    for i, u in enumerate(ubis[:24]):
        k, drl, lab = ref.score_and_assign(u, gv, 0.05, drl, lab, i)
        sa_n.append(k)
    out["sa_n"] = np.array(sa_n, np.int32)
    out["sa_drlv2"] = drl
    out["sa_labels"] = lab
    # adversarial boundary set
    u0 = ps.ubis[0]
    g_adv = adversarial_gv(u0, rng)
    specials = np.array([[np.nan, 0.1, 0.2], [np.inf, 0., 0.], [0., -np.inf, 1.],
                         [1e30, 1e30, -1e30], [3e15, 1., 2.], [0., 0., 0.]])
    g_adv = np.concatenate([g_adv, specials])
    out["adv_gv"] = g_adv
    out["adv_ubi"] = u0
    out["adv_counts"] = np.array([ref.score(u0, g_adv, t) for t in tols], np.int32)
    an, ad, au = [], [], []
    for t in tols:
        a, b, c = ref.score_and_refine(u0, g_adv[:-6], t)
        an.append(a); ad.append(b); au.append(c)
    out["adv_sar_n"] = np.array(an, np.int32)
    out["adv_sar_drlv2"] = np.array(ad)
    out["adv_sar_ubi"] = np.array(au)
    # singular / degenerate refinement: 0, 1, 2 peaks and coplanar peaks
    sing = []
    h_sets = [np.zeros((0, 3)), np.array([[1., 1, 1]]), np.array([[1., 1, 1], [2, 0, 0]]),
              np.array([[1., 1, 1], [2, 0, 0], [1, -1, -1], [3, 1, 1]])]
    for i, hset in enumerate(h_sets):
        g = hset @ np.linalg.inv(u0).T
        a, b, c = ref.score_and_refine(u0, g, 0.05)
        sing.append(np.concatenate([[a, b], c.ravel()]))
        out["sing%d_gv" % i] = g.reshape(-1, 3)
    out["sing_results"] = np.array(sing)
    return out


ADJ_PARAMS = ("distance", "y_center", "z_center", "tilt_x", "tilt_y", "tilt_z", "wavelength",
              "wedge", "chi", "t_x", "t_y", "t_z")
ADJ_STEPS = dict(distance=1e-2, y_center=1e-4, z_center=1e-4, tilt_x=1e-7, tilt_y=1e-7,
                 tilt_z=1e-7, wavelength=1e-8, wedge=1e-5, chi=1e-5, t_x=1e-3, t_y=1e-3,
                 t_z=1e-3)


def reference_loss(tr, s, f, omega, hkl, grain, ubis, pars):
    """0.5 * sum |UBI.g - h|^2 with g from the reference's numpy transform."""
    xyz = tr.compute_xyz_lab((s, f), **pars)
    om = omega * pars["omegasign"]
    tth, eta = tr.compute_tth_eta_from_xyz(xyz, om, t_x=pars["t_x"], t_y=pars["t_y"],
                                           t_z=pars["t_z"], wedge=pars["wedge"],
                                           chi=pars["chi"])
    g = tr.compute_g_vectors(tth, eta, om, pars["wavelength"], wedge=pars["wedge"],
                             chi=pars["chi"]).T
    r = np.einsum("nij,nj->ni", ubis[grain], g) - hkl
    return 0.5 * float((r * r).sum())


def cases_adjoint(tr):
    """Loss and central-difference gradients of the reference's forward model
    at a geometry away from the truth (cfg3-like tilts, wedge, chi, t)."""
    truth = synth.default_geometry(distance=152300., y_center=1024 + 3.7, z_center=1024 - 2.1,
                                   tilt_x=0.004, tilt_y=-0.002, tilt_z=0.006, wedge=0.01,
                                   chi=0.02, t_x=5., t_y=-3., t_z=2.)
    ps = synth.simulate(6, "Al", gmax=1.2, seed=21, geo=truth, sigma_px=0.3, sigma_om=0.02,
                        noise_frac=0.0, translation=(5., -3., 2.))
    idx, off = ps.grain_offsets()
    s, f, om, hkl = ps.s[idx], ps.f[idx], ps.omega[idx], ps.hkl[idx]
    grain = np.repeat(np.arange(len(off) - 1), np.diff(off))
    rng = np.random.default_rng(22)
    ubis = synth.perturb_ubis(ps.ubis, 0.05, 0.0005, rng)
    pars = dict(truth, distance=152000., y_center=1024., z_center=1024., tilt_x=0.001,
                tilt_y=0.0, tilt_z=0.002, wedge=0.0, chi=0.0, t_x=0., t_y=0., t_z=0.)
    L0 = reference_loss(tr, s, f, om, hkl, grain, ubis, pars)
    grad = []
    for name in ADJ_PARAMS:
        h = ADJ_STEPS[name]
        lp = reference_loss(tr, s, f, om, hkl, grain, ubis, dict(pars, **{name: pars[name] + h}))
        lm = reference_loss(tr, s, f, om, hkl, grain, ubis, dict(pars, **{name: pars[name] - h}))
        grad.append((lp - lm) / (2 * h))
    gu = []
    for (G, i, j) in [(0, 0, 0), (1, 1, 2), (3, 2, 1), (5, 0, 2)]:
        h = 1e-7
        up = ubis.copy(); up[G, i, j] += h
        um = ubis.copy(); um[G, i, j] -= h
        gu.append((reference_loss(tr, s, f, om, hkl, grain, up, pars) -
                   reference_loss(tr, s, f, om, hkl, grain, um, pars)) / (2 * h))
    return dict(adj_s=s, adj_f=f, adj_omega=om, adj_hkl=hkl, adj_offsets=off, adj_ubis=ubis,
                adj_params=np.array([pars[k] for k in ADJ_PARAMS]),
                adj_const=np.array([pars["y_size"], pars["z_size"], pars["omegasign"],
                                    pars["o11"], pars["o12"], pars["o21"], pars["o22"]]),
                adj_loss=np.array(L0), adj_grad_fd=np.array(grad),
                adj_grad_ubi_idx=np.array([(0, 0, 0), (1, 1, 2), (3, 2, 1), (5, 0, 2)]),
                adj_grad_ubi_fd=np.array(gu),
                adj_truth=np.array([truth[k] for k in ADJ_PARAMS]))


def load_fittrans2(ref_root):
    """k_to_g and d_XSXB_to_gv from the reference's ImageD11/sandbox/fittrans2.py
    (its module-level imports need matplotlib and numba, so only these
    function definitions are taken from the file and run)."""
    import ast
    path = os.path.join(ref_root, "ImageD11", "sandbox", "fittrans2.py")
    tree = ast.parse(open(path).read())
    fns = [n for n in tree.body
           if isinstance(n, ast.FunctionDef) and n.name in ("k_to_g", "d_XSXB_to_gv")]
    ns = {"np": np}
    exec(compile(ast.Module(body=fns, type_ignores=[]), path, "exec"), ns)
    return ns["k_to_g"], ns["d_XSXB_to_gv"]


def load_deriv(ref_root):
    """g_to_k and make_ax of the reference's src/deriv.c, compiled by
    ``make -C oracle deriv`` into oracle/_ref/libderiv_ref.so."""
    import ctypes
    so = os.path.join(REPO, "oracle", "_ref", "libderiv_ref.so")
    if not os.path.exists(so):
        import subprocess
        subprocess.check_call(["make", "-C", os.path.join(REPO, "oracle"), "deriv",
                               "REF=" + ref_root])
    lib = ctypes.CDLL(so)
    p = ctypes.POINTER(ctypes.c_double)
    lib.g_to_k.argtypes = [p, p, p, p, ctypes.c_double, p, p, p, p, p]
    lib.g_to_k.restype = ctypes.c_int
    lib.make_ax.argtypes = [p, p, p, p]
    lib.make_ax.restype = ctypes.c_int
    return lib


def cases_derivatives(tr, ref_root):
    """Hand-derived derivatives of the reference, for the adjoint tests:

    * dg/dt (the grain translation) of ImageD11/sandbox/fittrans2.py:39-77
      (d_XSXB_to_gv) on peaks computed through the reference's
      compute_xyz_lab and k_to_g with wedge and chi set;
    * theta and dtheta/dUB of src/deriv.c:38-53 (g_to_k's tth_calc[0:10])
      for the UB matrices and hkl of simulated grains."""
    import ctypes
    k_to_g, d_xsxb = load_fittrans2(ref_root)
    gvg = sys.modules["ImageD11.gv_general"]
    truth = synth.default_geometry(distance=152300., y_center=1024 + 3.7, z_center=1024 - 2.1,
                                   tilt_x=0.004, tilt_y=-0.002, tilt_z=0.006, wedge=0.3,
                                   chi=-0.2, t_x=5., t_y=-3., t_z=2.)
    ps = synth.simulate(3, "Al", gmax=1.2, seed=23, geo=truth, sigma_px=0.3, sigma_om=0.02,
                        noise_frac=0.0, translation=(5., -3., 2.))
    idx, off = ps.grain_offsets()
    s, f, om, hkl = ps.s[idx], ps.f[idx], ps.omega[idx], ps.hkl[idx]
    pars = dict(truth, t_x=4.0, t_y=-2.5, t_z=1.5)
    xyz = tr.compute_xyz_lab((s, f), **pars)
    omr = np.radians(om * pars["omegasign"])
    cw = gvg.chiwedge(pars["chi"], pars["wedge"])
    XS = k_to_g(xyz, np.cos(omr), np.sin(omr), cw)
    beam = np.zeros((3, len(om)))
    beam[0] = 1.0
    XB = k_to_g(beam, np.cos(omr), np.sin(omr), cw)
    g, dgdt = d_xsxb(XS, XB, pars["t_x"], pars["t_y"], pars["t_z"], pars["wavelength"])
    # the same g through the reference transform (a check of the frames)
    tth, eta = tr.compute_tth_eta_from_xyz(xyz, om * pars["omegasign"], t_x=pars["t_x"],
                                           t_y=pars["t_y"], t_z=pars["t_z"],
                                           wedge=pars["wedge"], chi=pars["chi"])
    gref = tr.compute_g_vectors(tth, eta, om * pars["omegasign"], pars["wavelength"],
                                wedge=pars["wedge"], chi=pars["chi"])
    assert np.abs(g - gref).max() < 1e-12
    # deriv.c: UB = inv(UBI) of each grain, reflections of its peaks
    lib = load_deriv(ref_root)
    D = ctypes.POINTER(ctypes.c_double)

    def arr(a):
        return np.ascontiguousarray(a, dtype=np.float64)

    eye = arr(np.eye(3).ravel())
    axis, bm, ax = arr([0., 0., 1.]), arr([1., 0., 0.]), np.zeros(19)
    lib.make_ax(eye.ctypes.data_as(D), axis.ctypes.data_as(D), bm.ctypes.data_as(D),
                ax.ctypes.data_as(D))
    ubs = np.array([np.linalg.inv(u) for u in ps.ubis])
    grain = np.repeat(np.arange(len(off) - 1), np.diff(off))
    theta = np.empty(len(hkl))
    dtheta = np.empty((len(hkl), 9))
    for k in range(len(hkl)):
        h4 = arr([hkl[k, 0], hkl[k, 1], hkl[k, 2], 1.0])
        ub = arr(ubs[grain[k]].ravel())
        gc, kc = np.zeros(3), np.zeros(3)
        tc, ec, oc = np.zeros(10), np.zeros(10), np.zeros(10)
        lib.g_to_k(h4.ctypes.data_as(D), ub.ctypes.data_as(D), ax.ctypes.data_as(D),
                   eye.ctypes.data_as(D), pars["wavelength"], gc.ctypes.data_as(D),
                   kc.ctypes.data_as(D), tc.ctypes.data_as(D), ec.ctypes.data_as(D),
                   oc.ctypes.data_as(D))
        theta[k] = tc[0]
        dtheta[k] = tc[1:10]
    return dict(der_s=s, der_f=f, der_omega=om, der_hkl=hkl, der_offsets=off,
                der_params=np.array([pars[k] for k in ADJ_PARAMS]),
                der_const=np.array([pars["y_size"], pars["z_size"], pars["omegasign"],
                                    pars["o11"], pars["o12"], pars["o21"], pars["o22"]]),
                der_g=g.T.copy(), der_dgdt=np.moveaxis(dgdt, 2, 0).copy(),
                der_ubs=ubs, der_theta=theta, der_dtheta=dtheta)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMAGED11_REF")
    if not ref_root:
        sys.exit("usage: make_golden.py /path/to/ImageD11 (or set IMAGED11_REF)")
    ref = Reference()
    tr = import_reference_transform(ref_root)
    assert ref.verify_rounding(20) == 0
    np.savez_compressed(os.path.join(HERE, "compute_gv.npz"), **cases_compute_gv(ref, tr))
    np.savez_compressed(os.path.join(HERE, "compute_xlylzl.npz"), **cases_xlylzl(ref, tr))
    np.savez_compressed(os.path.join(HERE, "scoring.npz"), **cases_scoring(ref))
    np.savez_compressed(os.path.join(HERE, "adjoint.npz"), **cases_adjoint(tr))
    np.savez_compressed(os.path.join(HERE, "derivatives.npz"), **cases_derivatives(tr, ref_root))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
