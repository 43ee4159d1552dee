"""Seeded synthetic 3DXRD peak sets (input generation for tests and benchmarks).

No dataset ships with the reference for this path, so workloads are simulated:
grains of a given unit cell with orientations uniform on SO(3), all allowed
reflections below a |g| cutoff, diffraction angles solved for a rotating
sample, spots projected onto a tilted flat detector, centroid noise and
uniform noise peaks added.  The forward model is the exact inverse of the
geometry that compute_gv / compute_xlylzl implement
(ImageD11 src/cdiffraction.c:112-224, ImageD11/transform.py:51-147):

  lab spot  xyz = R_det . (0, (f - y_center)*y_size, (s - z_center)*z_size)^T + (distance,0,0)
  origin      o = W . Omega(w)^T . t              W = chi.wedge matrix
  k           = (xyz - o)/|xyz - o| - x_hat) / wavelength
  g           = Omega(w) . W^T . k

Cell conventions follow ImageD11/unitcell.py:233-262 (Busing & Levy B
matrix; UBI = inv(U.B); h = UBI.g).  Reflection conditions: F (h,k,l all
even or all odd, ImageD11/unitcell.py:97-98), I (h+k+l even), and hcp
P6_3/mmc (l odd with h+2k = 3n absent).  Random orientations are normalised
Gaussian quaternions, as in ImageD11 test/test_indexing.py:10-27.

Everything here is numpy on the host and is used only to make inputs; the
product's kernels never call it.
"""
import math

import numpy as np

# ---------------------------------------------------------------- crystals --

def b_matrix(a, b, c, alpha=90.0, beta=90.0, gamma=90.0):
    """Busing & Levy B (reciprocal basis as columns), as ImageD11/unitcell.py:233-262."""
    ca, cb, cg = (math.cos(math.radians(x)) for x in (alpha, beta, gamma))
    G = np.array([[a * a, a * b * cg, a * c * cb],
                  [a * b * cg, b * b, b * c * ca],
                  [a * c * cb, b * c * ca, c * c]])
    gi = np.linalg.inv(G)
    astar, bstar, cstar = np.sqrt(np.diag(gi))
    alphas = math.degrees(math.acos(gi[1, 2] / bstar / cstar))
    betas = math.degrees(math.acos(gi[0, 2] / astar / cstar))
    gammas = math.degrees(math.acos(gi[0, 1] / astar / bstar))
    return np.array([[astar, bstar * math.cos(math.radians(gammas)),
                      cstar * math.cos(math.radians(betas))],
                     [0, bstar * math.sin(math.radians(gammas)),
                      -cstar * math.sin(math.radians(betas)) * ca],
                     [0, 0, 1.0 / c]])


CELLS = {
    # name: (a, b, c, alpha, beta, gamma, lattice)
    "Al": (4.05, 4.05, 4.05, 90., 90., 90., "F"),
    "Ti_hcp": (2.95, 2.95, 4.68, 90., 90., 120., "hcp"),
    "Ti_beta": (3.31, 3.31, 3.31, 90., 90., 90., "I"),
}


def allowed(h, k, l, lattice):
    if lattice == "F":
        return ((h % 2 == k % 2) & (k % 2 == l % 2))
    if lattice == "I":
        return (h + k + l) % 2 == 0
    if lattice == "hcp":
        return ~(((h + 2 * k) % 3 == 0) & (l % 2 == 1))
    return np.ones_like(h, dtype=bool)


def hkl_list(cell, gmax):
    """All allowed hkl (excluding 000) with |B.h| <= gmax, sorted by |g|."""
    a, b, c, al, be, ga, lat = CELLS[cell] if isinstance(cell, str) else cell
    B = b_matrix(a, b, c, al, be, ga)
    hm = int(gmax * max(a, b, c)) + 2
    r = np.arange(-hm, hm + 1)
    h, k, l = [x.ravel() for x in np.meshgrid(r, r, r, indexing="ij")]
    hkl = np.stack([h, k, l], 1)
    hkl = hkl[(hkl != 0).any(1) & allowed(h, k, l, lat)]
    gl = np.linalg.norm(hkl @ B.T, axis=1)
    keep = gl <= gmax
    hkl, gl = hkl[keep], gl[keep]
    o = np.argsort(gl, kind="stable")
    return hkl[o].astype(np.float64), B


def random_rotations(n, rng):
    """n rotation matrices uniform on SO(3) (normalised Gaussian quaternions)."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def axis_angle(axes, angles):
    """Rotation matrices about unit axes (n,3) by angles (n,) in radians."""
    axes = axes / np.linalg.norm(axes, axis=1)[:, None]
    x, y, z = axes.T
    c, s = np.cos(angles), np.sin(angles)
    C = 1 - c
    return np.stack([
        np.stack([c + x * x * C, x * y * C - z * s, x * z * C + y * s], -1),
        np.stack([y * x * C + z * s, c + y * y * C, y * z * C - x * s], -1),
        np.stack([z * x * C - y * s, z * y * C + x * s, c + z * z * C], -1),
    ], 1)


def perturb_ubis(ubis, angle_deg, strain, rng):
    """Rotate each UB by angle_deg about a random axis and apply a random
    symmetric strain of magnitude ~strain; returns the perturbed UBIs."""
    n = len(ubis)
    R = axis_angle(rng.normal(size=(n, 3)), np.full(n, math.radians(angle_deg)))
    e = rng.normal(size=(n, 3, 3)) * strain
    e = 0.5 * (e + np.transpose(e, (0, 2, 1)))
    ub = np.linalg.inv(ubis)
    ub2 = R @ (np.eye(3)[None] + e) @ ub
    return np.linalg.inv(ub2)


# ---------------------------------------------------------------- geometry --

def default_geometry(**kw):
    """ImageD11 parameter names (ImageD11/transform.py:656-673); lengths in um."""
    g = dict(distance=150000.0, y_center=1024.0, z_center=1024.0, y_size=75.0, z_size=75.0,
             tilt_x=0.0, tilt_y=0.0, tilt_z=0.0, o11=1.0, o12=0.0, o21=0.0, o22=-1.0,
             wavelength=0.2846, omegasign=1.0, wedge=0.0, chi=0.0,
             t_x=0.0, t_y=0.0, t_z=0.0, dim=2048)
    g.update(kw)
    return g


def detector_rotation_matrix(tilt_x, tilt_y, tilt_z):
    """R3(tilt_x) . R2(tilt_y) . R1(tilt_z), ImageD11/transform.py:51-82."""
    cz, sz = math.cos(tilt_z), math.sin(tilt_z)
    cy, sy = math.cos(tilt_y), math.sin(tilt_y)
    cx, sx = math.cos(tilt_x), math.sin(tilt_x)
    r1 = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1.]])
    r2 = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    r3 = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    return r3 @ r2 @ r1


def xlylzl_params(geo):
    """(p, r, dist) for compute_xlylzl: p = [s_cen, f_cen, s_size, f_size],
    r = detector_rotation . flip (ImageD11/transform.py:688-693)."""
    dmat = detector_rotation_matrix(geo["tilt_x"], geo["tilt_y"], geo["tilt_z"])
    fmat = np.array([[1, 0, 0], [0, geo["o22"], geo["o21"]], [0, geo["o12"], geo["o11"]]],
                    float)
    r = dmat @ fmat
    p = np.array([geo["z_center"], geo["y_center"], geo["z_size"], geo["y_size"]], float)
    dist = np.array([geo["distance"], 0.0, 0.0])
    return p, r, dist


def wedgechi(wedge, chi):
    """The chi.wedge matrix of ImageD11 src/cdiffraction.c:117-142 (row-major)."""
    sw, cw = math.sin(math.radians(wedge)), math.cos(math.radians(wedge))
    sc, cc = math.sin(math.radians(chi)), math.cos(math.radians(chi))
    W = np.array([[cw, 0.0, -sw], [0., 1.0, 0.], [sw, 0.0, cw]])
    C = np.array([[1., 0.0, 0.], [0., cc, -sc], [0., sc, cc]])
    return W @ C


def gv_numpy(xyz, omega, omegasign, wvln, wedge, chi, t):
    """g-vectors from lab positions (numpy; input generation only)."""
    M = wedgechi(wedge, chi)
    a = np.radians(omega * omegasign)
    so, co = np.sin(a), np.cos(a)
    t = np.asarray(t, float)
    u = np.stack([co * t[0] - so * t[1], so * t[0] + co * t[1], np.full_like(co, t[2])], 1)
    o = u @ M.T
    d = xyz - o
    d = d / np.linalg.norm(d, axis=1)[:, None]
    k = (d - np.array([1.0, 0, 0])) / wvln
    v = k @ M
    return np.stack([co * v[:, 0] + so * v[:, 1], -so * v[:, 0] + co * v[:, 1], v[:, 2]], 1)


def project_spots(g, t, geo):
    """Forward model: sample-frame g-vectors (n,3) of grains at translations
    t (n,3) -> (s, f, omega, valid) for both diffraction solutions (2n rows)."""
    lam = geo["wavelength"]
    M = wedgechi(geo["wedge"], geo["chi"])
    g0, g1, g2 = g.T
    A = M[0, 0] * g0 + M[0, 1] * g1
    Bc = M[0, 1] * g0 - M[0, 0] * g1
    gg = (g * g).sum(1)
    C = -lam * gg / 2 - M[0, 2] * g2
    Rab = np.hypot(A, Bc)
    q = np.where(Rab > 0, C / np.where(Rab > 0, Rab, 1), 2.0)
    ok = np.abs(q) <= 1
    phi = np.arctan2(Bc, A)
    dw = np.arccos(np.clip(q, -1, 1))
    out = []
    p, r, dist = xlylzl_params(geo)
    c1, c2 = r[:, 1], r[:, 2]
    nrm = np.cross(c1, c2)
    for w in (phi + dw, phi - dw):
        co, so = np.cos(w), np.sin(w)
        v = np.stack([co * g0 - so * g1, so * g0 + co * g1, g2], 1)
        k = v @ M.T
        dhat = lam * k + np.array([1.0, 0, 0])
        u = np.stack([co * t[:, 0] - so * t[:, 1], so * t[:, 0] + co * t[:, 1], t[:, 2]], 1)
        o = u @ M.T
        den = dhat @ nrm
        sfac = ((dist - o) @ nrm) / np.where(den != 0, den, 1)
        xyz = o + sfac[:, None] * dhat
        rel = xyz - dist
        v1, v2 = rel @ c1, rel @ c2
        f = v1 / p[3] + p[1]
        s = v2 / p[2] + p[0]
        om = np.degrees(w) / geo["omegasign"]
        om = np.mod(om, 360.0)
        valid = ok & (den != 0) & (sfac > 0) & (f >= 0) & (f < geo["dim"]) & (s >= 0) & \
            (s < geo["dim"])
        out.append((s, f, om, valid))
    s = np.concatenate([o[0] for o in out])
    f = np.concatenate([o[1] for o in out])
    om = np.concatenate([o[2] for o in out])
    valid = np.concatenate([o[3] for o in out])
    return s, f, om, valid


def xlylzl_numpy(s, f, geo):
    p, r, dist = xlylzl_params(geo)
    v1 = (f - p[1]) * p[3]
    v2 = (s - p[0]) * p[2]
    return v1[:, None] * r[:, 1][None] + v2[:, None] * r[:, 2][None] + dist[None]


# ------------------------------------------------------------------- scenes --

class PeakSet:
    """A simulated scan: spots (s, f, omega), their grain labels (-1 = noise),
    true UBIs, translations and the geometry; gv computed in numpy."""

    def __init__(self, s, f, omega, labels, ubis, translations, geo, gcut, cell):
        self.s, self.f, self.omega, self.labels = s, f, omega, labels
        self.ubis, self.translations, self.geo = ubis, translations, geo
        self.gcut, self.cell = gcut, cell
        self.xyz = xlylzl_numpy(s, f, geo)
        t = np.array([geo["t_x"], geo["t_y"], geo["t_z"]])
        self.gv = gv_numpy(self.xyz, omega, geo["omegasign"], geo["wavelength"], geo["wedge"],
                           geo["chi"], t)

    def __len__(self):
        return len(self.s)

    def grain_offsets(self):
        """CSR over grains after sorting peaks by label (noise peaks dropped)."""
        keep = self.labels >= 0
        o = np.argsort(self.labels[keep], kind="stable")
        lab = self.labels[keep][o]
        offsets = np.searchsorted(lab, np.arange(len(self.ubis) + 1))
        return np.nonzero(keep)[0][o], offsets.astype(np.int64)


def simulate(ngrains, cell="Al", gmax=1.0, seed=0, geo=None, sigma_px=0.5, sigma_om=0.05,
             noise_frac=0.10, per_grain_counts=None, translations_um=0.0, cells=None,
             translation=None):
    """Simulate a scan.  per_grain_counts (optional) keeps, for each grain, only
    its lowest-|g| spots up to that count (a per-grain |g| cutoff).
    translation (optional 3-vector) places every grain at that position
    (otherwise uniform in +-translations_um).  The returned PeakSet records
    each spot's true hkl (NaN for noise peaks)."""
    rng = np.random.default_rng(seed)
    geo = default_geometry() if geo is None else geo
    cells = cells if cells is not None else [cell] * ngrains
    U = random_rotations(ngrains, rng)
    trans = rng.uniform(-1, 1, size=(ngrains, 3)) * translations_um
    if translation is not None:
        trans = np.tile(np.asarray(translation, float), (ngrains, 1))
    cache = {}
    ubis = np.empty((ngrains, 3, 3))
    S, F, OM, LAB, HKL = [], [], [], [], []
    for name in sorted(set(cells)):
        if name not in cache:
            cache[name] = hkl_list(name, gmax)
        hkl, B = cache[name]
        idx = np.array([i for i in range(ngrains) if cells[i] == name])
        UB = U[idx] @ B
        ubis[idx] = np.linalg.inv(UB)
        g = np.einsum("nij,hj->nhi", UB, hkl)           # (n, H, 3)
        n, H = g.shape[:2]
        gl = np.broadcast_to(np.linalg.norm(hkl @ B.T, axis=1), (n, H))
        tt = np.repeat(trans[idx], H, axis=0)
        s, f, om, valid = project_spots(g.reshape(-1, 3), tt, geo)
        lab = np.tile(np.repeat(idx, H), 2)
        gsort = np.tile(gl.reshape(-1), 2)
        hk = np.tile(np.tile(hkl, (n, 1)), (2, 1))
        s, f, om, lab, gsort = s[valid], f[valid], om[valid], lab[valid], gsort[valid]
        hk = hk[valid]
        if per_grain_counts is not None:
            o = np.lexsort((gsort, lab))
            s, f, om, lab, hk = s[o], f[o], om[o], lab[o], hk[o]
            start = np.searchsorted(lab, lab, side="left")
            rank = np.arange(len(lab)) - start
            keep = rank < np.asarray(per_grain_counts)[lab]
            s, f, om, lab, hk = s[keep], f[keep], om[keep], lab[keep], hk[keep]
        S.append(s); F.append(f); OM.append(om); LAB.append(lab); HKL.append(hk)
    s, f, om, lab, hk = (np.concatenate(x) for x in (S, F, OM, LAB, HKL))
    s = s + rng.normal(size=len(s)) * sigma_px
    f = f + rng.normal(size=len(f)) * sigma_px
    om = om + rng.normal(size=len(om)) * sigma_om
    nn = int(round(len(s) * noise_frac))
    s = np.concatenate([s, rng.uniform(0, geo["dim"], nn)])
    f = np.concatenate([f, rng.uniform(0, geo["dim"], nn)])
    om = np.concatenate([om, rng.uniform(0, 360, nn)])
    lab = np.concatenate([lab, np.full(nn, -1)]).astype(np.int32)
    hk = np.concatenate([hk, np.full((nn, 3), np.nan)])
    perm = rng.permutation(len(s))
    out = PeakSet(s[perm], f[perm], om[perm], lab[perm], ubis, trans, geo, gmax, cell)
    out.hkl = hk[perm]
    return out


def grain_gvectors(counts, cell, rng, sigma=5e-4):
    """Per-grain g-vector sets without a detector: grain i (orientation uniform
    on SO(3)) keeps its counts[i] shortest allowed reflections (a per-grain |g|
    cutoff; hkl and -hkl both), g = U.B.hkl plus Gaussian noise of sigma
    (1/A) per component.  Returns (gv (n,3) sorted by grain, offsets
    (ngrains+1,) int64, true UBIs (ngrains,3,3))."""
    counts = np.asarray(counts, dtype=np.int64)
    a, b, c, al, be, ga, lat = CELLS[cell]
    B = b_matrix(a, b, c, al, be, ga)
    gmax = 0.5
    while True:  # reflections enough for the largest grain
        hkl, _ = hkl_list(cell, gmax)
        if len(hkl) >= counts.max():
            break
        gmax *= 1.25
    U = random_rotations(len(counts), rng)
    UB = U @ B
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    gv = np.empty((int(offsets[-1]), 3))
    for i, k in enumerate(counts):
        gv[offsets[i]:offsets[i + 1]] = hkl[:k] @ UB[i].T
    gv += rng.normal(size=gv.shape) * sigma
    return gv, offsets, np.linalg.inv(UB)


def trial_ubis(true_ubis, ntrial, frac_true, angle_deg, rng, cell="Al"):
    """Trial UBIs: frac_true of them perturbed copies of true UBIs, the rest
    uniformly random orientations of the same cell."""
    nt = int(round(ntrial * frac_true))
    pick = rng.integers(0, len(true_ubis), nt)
    t = perturb_ubis(true_ubis[pick], angle_deg, 0.0, rng)
    a, b, c, al, be, ga, lat = CELLS[cell]
    B = b_matrix(a, b, c, al, be, ga)
    U = random_rotations(ntrial - nt, rng)
    r = np.linalg.inv(U @ B)
    out = np.concatenate([t, r])
    return out[rng.permutation(ntrial)]
