"""Batched FP32-screened scoring / refinement vs the oracle and the golden vectors.

Counts are bit-exact (the FP64 recheck band makes every assignment decision
identical to the reference's); refined UBIs agree to the rounding of the sum
order.  Summed drlv2 of the counted pairs comes from the FP32 screening values:
each term is within the kernel's proven band of the FP64 value, so the sum is
checked against n * band + 1e-6 relative (FP32 accumulation).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UBI_RTOL = 1e-11
SUM_RTOL = 1e-6


def screening_band(ubis, gv, tol):
    """The kernel's per-pair bound on |drlv2_fp32 - drlv2_fp64| (score_batch.cu)."""
    eps = 2.0 ** -24
    ok = np.isfinite(gv).all(1) & (np.abs(gv).max(1) <= 1024)
    gmax = np.abs(gv[ok]).max()
    smax = np.abs(ubis).sum(-1).max() * (1 + 1e-6)
    E = 6 * eps * smax * gmax
    return 1.25 * (3 * E * (2 * (tol + 1e-3) + E) + 4 * eps * (tol * tol + 0.01))


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


def test_golden_counts(B, golden, oracle, cuda):
    d = golden["scoring"]
    gs = B.GvecSet(d["sc_gv"])
    c = B.score_batch(d["sc_ubis"], gs, d["sc_tols"]).cpu().numpy()
    assert np.array_equal(c, d["sc_counts"])
    c64 = B.score_many_fp64(d["sc_ubis"], gs, d["sc_tols"]).cpu().numpy()
    assert np.array_equal(c64, d["sc_counts"])


def test_adversarial_and_special_g(B, golden, oracle, cuda):
    d = golden["scoring"]
    gs = B.GvecSet(d["adv_gv"])
    ubis = np.concatenate([d["adv_ubi"][None], d["sc_ubis"][:7]])
    c = B.score_batch(ubis, gs, d["sc_tols"]).cpu().numpy()
    assert np.array_equal(c[0], d["adv_counts"])
    assert np.array_equal(c, oracle.score_many(ubis, d["adv_gv"], d["sc_tols"]))


def test_scene_counts_and_sums(B, oracle, scene, cuda):
    ps, ubis = scene
    tols = [0.02, 0.05, 0.1]
    gs = B.GvecSet(ps.gv)
    c, s = B.score_batch(ubis, gs, tols, sums=True)
    c = c.cpu().numpy()
    ref = oracle.score_many(ubis, ps.gv, tols)
    assert np.array_equal(c, ref)
    assert np.array_equal(B.score_many_fp64(ubis, gs, tols).cpu().numpy(), ref)
    s = s.cpu().numpy()
    for i in range(0, len(ubis), 37):
        for j, t in enumerate(tols):
            n, mean, _ = oracle.score_and_refine(ubis[i], ps.gv, t)
            assert n == c[i, j]
            bound = n * screening_band(ubis, ps.gv, t) + SUM_RTOL * mean * n
            assert abs(s[i, j] - mean * n) <= bound
    # order-free (fixed-point) accumulation: the same sums, bit for bit
    c2, s2 = B.score_batch(ubis, gs, tols, sums=True)
    assert np.array_equal(c2.cpu().numpy(), c) and np.array_equal(s2.cpu().numpy(), s)
    nrecheck, nfallback = B.score_batch.last_workspace.stats()
    assert nfallback == 0
    assert nrecheck < 1e-3 * len(ubis) * len(ps.gv)


def test_ragged_sizes(B, oracle, scene, cuda):
    ps, ubis = scene
    for m, n in [(1, 1), (1, 1023), (3, 1025), (1025, 777), (257, 5000)]:
        g = ps.gv[:n]
        u = ubis[:m]
        gs = B.GvecSet(g)
        c = B.score_batch(u, gs, [0.05, 0.1]).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(u, g, [0.05, 0.1])), (m, n)


def test_empty(B, cuda):
    gs = B.GvecSet(np.zeros((0, 3)))
    c = B.score_batch(np.eye(3)[None] * 4.05, gs, [0.1]).cpu().numpy()
    assert c.shape == (1, 1) and c[0, 0] == 0
    gs = B.GvecSet(np.ones((10, 3)))
    c = B.score_batch(np.zeros((0, 3, 3)), gs, [0.1])
    assert c.shape == (0, 1)


def test_fallback_ubis_and_large_tol(B, oracle, scene, cuda):
    ps, ubis = scene
    g = ps.gv[:20000]
    u = ubis[:40].copy()
    u[3] *= 1e5                      # S*gmax beyond the FP32 argument -> exact FP64
    u[5, 1, 1] = np.nan              # non-finite UBI
    u[7] = 0.0                       # all h = 0: every g counted
    gs = B.GvecSet(g)
    c = B.score_batch(u, gs, [0.05, 0.1]).cpu().numpy()
    assert np.array_equal(c, oracle.score_many(u, g, [0.05, 0.1]))
    nrecheck, nfallback = B.score_batch.last_workspace.stats()
    assert nfallback == 2
    c = B.score_batch(u, gs, [0.1, 0.47]).cpu().numpy()   # 0.47: all pairs in FP64
    assert np.array_equal(c, oracle.score_many(u, g, [0.1, 0.47]))


def test_refine_batch_matches_iterated_reference(B, oracle, scene, cuda):
    from imaged11_b200 import synth
    ps, _ = scene
    rng = np.random.default_rng(5)
    u0 = synth.perturb_ubis(ps.ubis[:50], 0.1, 0.001, rng)
    gs = B.GvecSet(ps.gv)
    u, npk, mean = B.refine_batch(u0.copy(), gs, 0.05, iters=3)
    u = u.cpu().numpy()
    npk = npk.cpu().numpy()
    mean = mean.cpu().numpy()
    for i in range(len(u0)):
        uu = u0[i].copy()
        for _ in range(3):
            n, m, uu = oracle.score_and_refine(uu, ps.gv, 0.05)
        assert npk[i] == n
        assert abs(mean[i] - m) <= 1e-12 * m
        assert np.abs(u[i] - uu).max() <= UBI_RTOL * np.abs(uu).max()


def test_random_sweep(B, oracle, cuda):
    """Random cells, orientations, g clouds and tolerances (g on rounding
    half-points included) against the oracle, through the FP32 screening."""
    rng = np.random.default_rng(78)
    for trial in range(24):
        n = int(rng.integers(1, 6000))
        gv = rng.normal(size=(n, 3)) * rng.uniform(0.2, 2.0)
        m = int(rng.integers(1, 700))
        ubis = np.empty((m, 3, 3))
        for i in range(m):
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            ubis[i] = np.diag(rng.uniform(1.5, 12.0, 3)) @ q.T
        if trial % 3 == 1:
            gv[: n // 3] = np.linalg.solve(ubis[0], (rng.integers(-5, 5, (n // 3, 3)) + 0.5).T).T
        tols = sorted(rng.uniform(0.001, 0.6, int(rng.integers(1, 5))).tolist())
        c = B.score_batch(ubis, B.GvecSet(gv), tols).cpu().numpy()
        assert np.array_equal(c, oracle.score_many(ubis, gv, tols)), trial
