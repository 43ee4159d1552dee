"""Scoring through the reciprocal-space cell index vs the oracle and the
golden vectors, by both methods: per-box lookups ("walk", every candidate
pair evaluated in the reference's FP64 arithmetic) and the binned join
("bins", FP32 screening with the proven FP64 recheck band).

Counts are bit-exact: the lookup boxes are conservative, so the counted set
is the reference's.  Sums of drlv2 are FP64 sums in another order than the
reference's loop: 1e-12 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12
METHODS = ["walk", "bins"]


@pytest.fixture(scope="module")
def B():
    from imaged11_b200 import batch
    return batch


@pytest.fixture(scope="module")
def scene():
    from imaged11_b200 import synth
    ps = synth.simulate(120, "Al", gmax=1.3, seed=31, noise_frac=0.10)
    rng = np.random.default_rng(32)
    ubis = synth.trial_ubis(ps.ubis, 1500, 0.1, 0.5, rng)
    return ps, ubis


@pytest.mark.parametrize("method", METHODS)
def test_golden_counts(B, golden, method, cuda):
    d = golden["scoring"]
    grid = B.GvecGrid(d["sc_gv"])
    c = B.score_grid(d["sc_ubis"], grid, d["sc_tols"], method=method).cpu().numpy()
    assert np.array_equal(c, d["sc_counts"])


@pytest.mark.parametrize("method", METHODS)
def test_adversarial_and_special_g(B, golden, oracle, method, cuda):
    d = golden["scoring"]
    grid = B.GvecGrid(d["adv_gv"])
    st = grid.stats()
    assert st["regular"] + st["special"] == len(d["adv_gv"])
    ubis = np.concatenate([d["adv_ubi"][None], d["sc_ubis"][:7]])
    c = B.score_grid(ubis, grid, d["sc_tols"], method=method).cpu().numpy()
    assert np.array_equal(c[0], d["adv_counts"])
    assert np.array_equal(c, oracle.score_many(ubis, d["adv_gv"], d["sc_tols"]))


@pytest.mark.parametrize("method", METHODS)
def test_scene_counts_and_sums(B, oracle, scene, method, cuda):
    ps, ubis = scene
    tols = [0.02, 0.05, 0.1]
    grid = B.GvecGrid(ps.gv)
    c, s = B.score_grid(ubis, grid, tols, sums=True, method=method)
    c = c.cpu().numpy()
    s = s.cpu().numpy()
    assert np.array_equal(c, oracle.score_many(ubis, ps.gv, tols))
    st = grid.stats()
    assert st["fallback_ubis"] == 0
    assert st["pairs_tested"] < 0.05 * len(ubis) * len(ps.gv)   # the point of the index
    for i in range(0, len(ubis), 37):
        for j, t in enumerate(tols):
            n, mean, _ = oracle.score_and_refine(ubis[i], ps.gv, t)
            assert n == c[i, j]
            # bins: each partial sum rounded to the fixed-point step (n terms
            # below tmax^2 in 2^62 steps)
            step = 0.0 if method == "walk" else 2.0 ** -(62 - np.ceil(np.log2(
                len(ps.gv) * max(tols) ** 2)))
            assert abs(s[i, j] - mean * n) <= SUM_RTOL * mean * n + n * step + 1e-300
    c2, s2 = B.score_grid(ubis, grid, tols, sums=True, method=method)
    assert np.array_equal(c2.cpu().numpy(), c)
    # fixed-order sums (walk) and fixed-point order-free sums (bins): the same bits
    assert np.array_equal(s2.cpu().numpy(), s)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("cell,xsub", [(0.004, 4), (0.03, 1), (0.03, 16), (0.25, 3),
                                       (1.0, 4)])
def test_cell_sizes(B, oracle, scene, cell, xsub, method, cuda):
    ps, ubis = scene
    u = ubis[:300]
    grid = B.GvecGrid(ps.gv, cell=cell, xsub=xsub)
    if method == "bins" and not B.bins_fit(grid):
        with pytest.raises(ValueError):
            B.score_grid(u, grid, [0.05, 0.1], method=method)
        method = None            # the default takes the lookup scorer for this grid
    c = B.score_grid(u, grid, [0.05, 0.1], method=method).cpu().numpy()
    assert np.array_equal(c, oracle.score_many(u, ps.gv, [0.05, 0.1])), cell


@pytest.mark.parametrize("method", METHODS)
def test_ragged_and_empty(B, oracle, scene, method, cuda):
    ps, ubis = scene
    for m, n in [(1, 1), (1, 1023), (3, 1025), (1025, 777), (257, 5000)]:
        g = ps.gv[:n]
        u = ubis[:m]
        c = B.score_grid(u, B.GvecGrid(g), [0.05, 0.1], method=method).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(u, g, [0.05, 0.1])), (m, n)
    c = B.score_grid(np.eye(3)[None] * 4.05, B.GvecGrid(np.zeros((0, 3))), [0.1],
                     method=method).cpu().numpy()
    assert c.shape == (1, 1) and c[0, 0] == 0
    c = B.score_grid(np.zeros((0, 3, 3)), B.GvecGrid(np.ones((10, 3))), [0.1], method=method)
    assert c.shape == (0, 1)


@pytest.mark.parametrize("method", METHODS)
def test_plain_scan_ubis_and_large_tols(B, oracle, scene, method, cuda):
    ps, ubis = scene
    g = ps.gv[:20000]
    u = ubis[:40].copy()
    u[3] *= 1e5                      # many more candidate hkl than g
    u[5, 1, 1] = np.nan              # non-finite
    u[7] = 0.0                       # singular: every g has h = 0
    u[9] = np.diag([1e4, 1.0, 1e-4]) # condition number 1e8
    grid = B.GvecGrid(g)
    c = B.score_grid(u, grid, [0.05, 0.1], method=method).cpu().numpy()
    assert np.array_equal(c, oracle.score_many(u, g, [0.05, 0.1]))
    assert grid.stats()["fallback_ubis"] == 4
    for tols in ([0.1, 0.47], [0.5, 0.9], [3.0]):
        c = B.score_grid(u, grid, tols).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(u, g, tols)), tols


@pytest.mark.parametrize("method", METHODS)
def test_matches_score_batch(B, scene, method, cuda):
    ps, ubis = scene
    tols = [0.01, 0.03, 0.07, 0.2]
    a = B.score_grid(ubis, B.GvecGrid(ps.gv), tols, method=method).cpu().numpy()
    b = B.score_batch(ubis, B.GvecSet(ps.gv), tols).cpu().numpy()
    assert np.array_equal(a, b)


def test_refine_grid_matches_iterated_reference(B, oracle, scene, cuda):
    from imaged11_b200 import synth
    ps, _ = scene
    rng = np.random.default_rng(5)
    u0 = synth.perturb_ubis(ps.ubis[:50], 0.1, 0.001, rng)
    u0 = np.concatenate([u0, np.zeros((1, 3, 3))])       # singular: plain scan, unchanged
    grid = B.GvecGrid(ps.gv)
    u, npk, mean = B.refine_grid(u0.copy(), grid, 0.05, iters=3)
    u, npk, mean = u.cpu().numpy(), npk.cpu().numpy(), mean.cpu().numpy()
    for i in range(len(u0)):
        uu = u0[i].copy()
        for _ in range(3):
            n, m, uu = oracle.score_and_refine(uu, ps.gv, 0.05)
        assert npk[i] == n
        assert abs(mean[i] - m) <= 1e-12 * m
        assert np.abs(u[i] - uu).max() <= 1e-11 * max(np.abs(uu).max(), 1e-300)
    ub, nb, mb = B.refine_batch(u0.copy(), B.GvecSet(ps.gv), 0.05, iters=3)
    assert np.array_equal(nb.cpu().numpy(), npk)


def test_refine_grid_special_g(B, golden, oracle, cuda):
    d = golden["scoring"]
    gv = d["adv_gv"]
    u0 = np.concatenate([d["adv_ubi"][None], d["sc_ubis"][:5]])
    grid = B.GvecGrid(gv)
    assert grid.stats()["special"] > 0
    u, npk, mean = B.refine_grid(u0.copy(), grid, 0.1, iters=2)
    u, npk, mean = u.cpu().numpy(), npk.cpu().numpy(), mean.cpu().numpy()
    for i in range(len(u0)):
        uu = u0[i].copy()
        for _ in range(2):
            n, m, uu = oracle.score_and_refine(uu, gv, 0.1)
        assert npk[i] == n
        assert abs(mean[i] - m) <= 1e-12 * m
        assert np.abs(u[i] - uu).max() <= 1e-11 * np.abs(uu).max()


def test_random_sweep(B, oracle, cuda):
    """Random cells, orientations, g clouds and tolerances (including ones above
    0.5 and g on the rounding half-points) against the oracle."""
    rng = np.random.default_rng(77)
    for trial in range(24):
        n = int(rng.integers(1, 6000))
        gv = rng.normal(size=(n, 3)) * rng.uniform(0.2, 2.0)
        if trial % 4 == 1:                       # a lattice's g plus noise
            a = rng.uniform(2.0, 9.0)
            hkl = rng.integers(-6, 7, size=(n, 3)).astype(float)
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            gv = (hkl / a) @ q.T + rng.normal(scale=1e-3, size=(n, 3))
        m = int(rng.integers(1, 300))
        ubis = np.empty((m, 3, 3))
        for i in range(m):
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            ubis[i] = np.diag(rng.uniform(1.5, 12.0, 3)) @ q.T
        if trial % 4 == 2:                       # h exactly on half-integers for some g
            gv[: n // 3] = np.linalg.solve(ubis[0], (rng.integers(-5, 5, (n // 3, 3)) + 0.5).T).T
        tols = sorted(rng.uniform(0.001, 0.7, int(rng.integers(1, 5))).tolist())
        c = B.score_grid(ubis, B.GvecGrid(gv), tols).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(ubis, gv, tols)), trial


def test_bins_random_sweep(B, oracle, cuda):
    """The binned join on random cells, orientations, g clouds (lattice g with
    noise, g on rounding half-points) and tolerances below 0.4."""
    rng = np.random.default_rng(78)
    for trial in range(24):
        n = int(rng.integers(1, 6000))
        gv = rng.normal(size=(n, 3)) * rng.uniform(0.2, 2.0)
        if trial % 3 == 1:
            a = rng.uniform(2.0, 9.0)
            hkl = rng.integers(-6, 7, size=(n, 3)).astype(float)
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            gv = (hkl / a) @ q.T + rng.normal(scale=1e-3, size=(n, 3))
        m = int(rng.integers(1, 300))
        ubis = np.empty((m, 3, 3))
        for i in range(m):
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            ubis[i] = np.diag(rng.uniform(1.5, 12.0, 3)) @ q.T
        if trial % 3 == 2:
            gv[: n // 3] = np.linalg.solve(ubis[0], (rng.integers(-5, 5, (n // 3, 3)) + 0.5).T).T
        tols = sorted(rng.uniform(0.001, 0.399, int(rng.integers(1, 5))).tolist())
        grid = B.GvecGrid(gv, cell=float(rng.uniform(0.01, 0.2)) if trial % 2 else None)
        if not B.bins_fit(grid):
            grid = B.GvecGrid(gv)
        c = B.score_grid(ubis, grid, tols, method="bins").cpu().numpy()
        assert np.array_equal(c, oracle.score_many(ubis, gv, tols)), trial


def test_bins_workspace_ranges(B, oracle, scene, cuda):
    """A workspace holding only part of the boxes: the UBIs run in ranges,
    with the same counts; too small for one UBI's boxes is an error."""
    from imaged11_b200._lib import ID11BError
    ps, ubis = scene
    u = ubis[:200]
    tols = [0.02, 0.05, 0.1]
    grid = B.GvecGrid(ps.gv)
    full = B.score_grid(u, grid, tols, method="bins").cpu().numpy()
    assert np.array_equal(full, oracle.score_many(u, ps.gv, tols))
    est = B.bins_box_estimate(u, grid, 0.1)
    for frac in (0.5, 0.13):
        ws = B.BinsWorkspace(len(u), grid, int(est * frac))
        c = B.score_grid(u, grid, tols, method="bins", workspace=ws).cpu().numpy()
        assert np.array_equal(c, full), frac
    with pytest.raises(ID11BError):
        B.score_grid(u, grid, tols, method="bins", workspace=B.BinsWorkspace(len(u), grid, 10))


def test_bins_rejects_large_tolerances(B, scene, cuda):
    ps, ubis = scene
    with pytest.raises(Exception):
        B.score_grid(ubis[:4], B.GvecGrid(ps.gv[:100]), [0.1, 0.4], method="bins")


def test_bins_unsorted_tolerances_and_large_hkl(B, oracle, scene, cuda):
    """The join counts with the tolerances sorted and writes each count (and
    sum) back to the caller's column: unsorted and repeated tolerances give the
    reference's counts column by column, and sums equal to the lookup's to the
    fixed-point step.  Cells elongated along one axis put h near +-250 (the
    record's limit is 255) through the join, the widest FMA-chain error bound."""
    ps, ubis = scene
    tols = [0.1, 0.05, 0.35, 0.05]
    grid = B.GvecGrid(ps.gv)
    c, s = B.score_grid(ubis[:400], grid, tols, sums=True, method="bins")
    cw, sw = B.score_grid(ubis[:400], grid, tols, sums=True, method="walk")
    ref = oracle.score_many(ubis[:400], ps.gv, tols)
    assert np.array_equal(c.cpu().numpy(), ref) and np.array_equal(cw.cpu().numpy(), ref)
    step = 2.0 ** -(62 - np.ceil(np.log2(len(ps.gv) * max(tols) ** 2)))
    diff = np.abs(s.cpu().numpy() - sw.cpu().numpy())
    assert np.all(diff <= 1e-12 * sw.cpu().numpy() + ref * step), diff.max()
    rng = np.random.default_rng(79)
    g = rng.normal(size=(400000, 3))
    g *= (1.5 * rng.uniform(size=(len(g), 1)) ** (1 / 3)) / np.linalg.norm(g, axis=1)[:, None]
    grid = B.GvecGrid(g)   # more g than the elongated cells' candidate hkl
    big = np.empty((60, 3, 3))
    G = grid.gmax * (1 + 1e-6)       # the cube that bounds every |hkl| of the plan
    for i in range(len(big)):
        th, ph = rng.uniform(0, 2 * np.pi), rng.uniform(-0.05, 0.05)
        rx = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
        rz = np.array([[np.cos(ph), -np.sin(ph), 0], [np.sin(ph), np.cos(ph), 0], [0, 0, 1]])
        m = (rz @ rx).T                                   # rows: the cell's axes
        s0 = rng.uniform(0.85, 0.99) * 253.0 / (G * np.abs(m[0]).sum())
        big[i] = np.diag([s0, *rng.uniform(2.0, 4.0, 2)]) @ m
    hmax = np.abs(np.einsum("mij,nj->mni", big[:8], g[:20000])).max()
    assert 150 < hmax < 255
    for t in ([0.3, 0.1, 0.2], [0.05]):
        c = B.score_grid(big, grid, t, method="bins").cpu().numpy()
        assert grid.stats()["fallback_ubis"] == 0
        assert np.array_equal(c, oracle.score_many(big, g, t)), t
        assert c[:, 0].sum() > 0


def _snap_to_cell_faces(grid, g, rng):
    """g moved to the nearest face of the index's cells in each coordinate
    (x faces every cs / xsub, y and z every cs, from the cube's corner lo),
    then one ulp down, left, or one ulp up, at random per coordinate."""
    lo = -(grid.gmax * (1. + 1e-6) + 1e-300)
    side = np.array([grid.cs / grid.xsub, grid.cs, grid.cs])
    q = lo + np.round((g - lo) / side) * side
    which = rng.integers(0, 3, size=g.shape)
    q = np.where(which == 1, np.nextafter(q, -np.inf),
                 np.where(which == 2, np.nextafter(q, np.inf), q))
    return np.clip(q, -grid.gmax, grid.gmax)


@pytest.mark.parametrize("method", METHODS)
def test_g_on_cell_faces(B, oracle, scene, method, cuda):
    """g-vectors on the faces of the cells (and one ulp either side): the build
    and every query take a g's cell from one monotone function, and the boxes
    are widened past their rounding, so counts there are the reference's."""
    import torch
    ps, ubis = scene
    rng = np.random.default_rng(31)
    for cell, xsub in ((0.03, 4), (0.05, 1)):
        grid = B.GvecGrid(ps.gv[:300000], cell=cell, xsub=xsub)
        q = _snap_to_cell_faces(grid, ps.gv[:300000], rng)
        grid.gv.copy_(torch.from_numpy(q))
        grid.refresh()
        assert grid.stats()["special"] < 0.01 * len(q)
        tols = [0.05, 0.1, 0.2]
        c = B.score_grid(ubis[:300], grid, tols, method=method).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(ubis[:300], q, tols)), (cell, xsub)
        assert c[:, 1].sum() > 1000


@pytest.mark.parametrize("method", METHODS)
def test_g_outside_the_built_bounds(B, oracle, scene, method, cuda):
    """A rebuild into the same shape after the g-vectors moved (refresh) keeps
    the cube and rmax of the first build: g now outside them join the list
    scored by a plain scan, so no box misses them and counts stay exact."""
    import torch
    ps, ubis = scene
    g = ps.gv[:200000]
    grid = B.GvecGrid(g)
    assert grid.stats()["special"] == 0
    moved = g * 1.08
    grid.gv.copy_(torch.from_numpy(moved))
    grid.refresh()
    st = grid.stats()
    outside = (np.abs(moved).max(axis=1) > grid.gmax) | \
        (np.linalg.norm(moved, axis=1) > grid.rmax)
    assert outside.sum() > 200 and st["special"] >= 0.99 * outside.sum()
    assert st["regular"] + st["special"] == len(g)
    tols = [0.05, 0.2]
    c = B.score_grid(ubis[:300], grid, tols, method=method).cpu().numpy()
    assert np.array_equal(c, oracle.score_many(ubis[:300], moved, tols))


def test_bins_more_ubis_than_a_box_record_holds(B, oracle, scene, cuda):
    """A box record holds its UBI's index within a range of 2^20 UBIs:
    1,053,576 UBIs are joined in two ranges, and every UBI's counts are the
    reference's."""
    ps, _ = scene
    g = ps.gv[:4000]
    rng = np.random.default_rng(7)
    m = (1 << 20) + 5000
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    a, b, c, d = q.T
    rot = np.stack([np.stack([1 - 2 * (c * c + d * d), 2 * (b * c - a * d), 2 * (b * d + a * c)], -1),
                    np.stack([2 * (b * c + a * d), 1 - 2 * (b * b + d * d), 2 * (c * d - a * b)], -1),
                    np.stack([2 * (b * d - a * c), 2 * (c * d + a * b), 1 - 2 * (b * b + c * c)], -1)],
                   1)
    ubis = rng.uniform(0.8, 1.6, size=(m, 1, 1)) * rot    # small cells: few boxes each
    grid = B.GvecGrid(g)
    tols = [0.1, 0.25]
    cnt = B.score_grid(ubis, grid, tols, method="bins").cpu().numpy()
    assert grid.stats()["fallback_ubis"] == 0
    assert np.array_equal(cnt, oracle.score_many(ubis, g, tols))
