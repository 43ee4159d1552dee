"""Launch-shape autotuner: every candidate tile gives the oracle's counts, the
tuned shape is cached and reused, and the refinement tuner leaves results
unchanged (to the rounding of the summation order)."""
import json

import numpy as np
import pytest


@pytest.fixture
def tune(monkeypatch):
    try:
        from imaged11_b200 import tune as t
    except ImportError as e:  # library not built
        pytest.skip(str(e))
    t.clear()
    yield t
    t.clear()


def test_cache_buckets_and_roundtrip(tune, monkeypatch, tmp_path):
    monkeypatch.setattr(tune, "_device_name", lambda: "dev0")
    assert tune.score_tile(1000, 5000, 3) is None
    tune._cache[tune.score_key(1000, 5000, 3)] = [2, 7]
    # same power-of-two bucket -> same entry; other ntol / bucket -> none
    assert tune.score_tile(1024, 4097, 3) == (2, 7)
    assert tune.score_tile(1025, 5000, 3) is None
    assert tune.score_tile(1000, 5000, 2) is None
    tune._cache[tune.refine_key(2000, 800000)] = 32
    assert tune.refine_threads(1500, 1000000) == 32
    p = tmp_path / "tune.json"
    tune.save(str(p))
    assert json.loads(p.read_text())["score|dev0|1024|8192|3"] == [2, 7]
    tune.clear()
    assert tune.score_tile(1000, 5000, 3) is None
    tune.load(str(p))
    assert tune.score_tile(1000, 5000, 3) == (2, 7)


def test_halo_cell_factor(tune):
    """The smallest cell side with a one-row join halo: W + 2 eps over the
    default side, W the largest widened box half width of the UBIs the join
    takes, computed here independently for rotated cubic cells."""
    import torch

    class Base:
        cs, gmax, n = 0.03, 1.5, 100000

    rng = np.random.default_rng(3)
    a = np.array([4.05, 3.0, 5.5])
    ubis = np.empty((3, 3, 3))
    for i in range(3):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        ubis[i] = a[i] * q
    tol = 0.1
    G = Base.gmax * (1 + 1e-6)
    W = 0.0
    for u in ubis:
        ub = np.linalg.inv(u)
        hm = np.ceil(np.abs(u).sum(axis=1) * G + 1.0)
        w = (tol + 1e-6) * np.linalg.norm(ub, axis=1) * (1 + 1e-9) + \
            4 * 2.0 ** -24 * hm.max() * np.abs(ub).sum(axis=1)
        W = max(W, w.max())
    want = (W + 4e-5 * (1 + G)) * (1 + 1e-3) / Base.cs
    got = tune.halo_cell_factor(torch.tensor(ubis), Base, tol)
    assert got == pytest.approx(want, rel=1e-12)
    assert got == pytest.approx(0.1 / 3.0 / Base.cs, rel=0.01)  # the smallest cell dominates
    assert tune.halo_cell_factor(torch.tensor(ubis), Base, 0.2) > got
    # UBIs the join does not take are left out: singular, or more candidate hkl than g
    big = ubis.copy()
    big[1] = 0.0
    big[2] *= 100.0
    assert tune.halo_cell_factor(torch.tensor(big), Base, tol) == pytest.approx(
        tune.halo_cell_factor(torch.tensor(ubis[:1]), Base, tol), rel=1e-12)
    assert tune.halo_cell_factor(torch.tensor(ubis[:0]), Base, tol) is None


@pytest.mark.gpu
def test_every_tile_exact_and_cached(tune, oracle, cuda):
    from imaged11_b200 import batch, synth
    ps = synth.simulate(60, "Al", gmax=1.2, seed=51, noise_frac=0.1)
    rng = np.random.default_rng(52)
    ubis = synth.trial_ubis(ps.ubis, 1300, 0.1, 0.5, rng)
    tols = [0.02, 0.05, 0.1]
    ref = oracle.score_many(ubis, ps.gv, tols)
    gs = batch.GvecSet(ps.gv)
    cands = tune.score_candidates(len(ubis), gs.n)
    assert {r for r, _ in cands} == {2, 4}
    for tile in cands + [(2, 1), (4, 10 ** 6)]:   # gsplit clamped to one tile per CTA
        c = batch.score_batch(ubis, gs, tols, tile=tile).cpu().numpy()
        assert np.array_equal(c, ref), tile
    best, table = tune.tune_score(ubis, gs, tols, reps=1)
    assert len(table) == len(cands) and best in cands
    assert tune.score_tile(len(ubis), gs.n, 3) == best
    assert np.array_equal(batch.score_batch(ubis, gs, tols).cpu().numpy(), ref)


@pytest.mark.gpu
def test_bad_tile_rejected(tune, cuda):
    from imaged11_b200 import batch
    from imaged11_b200._lib import ID11BError
    gs = batch.GvecSet(np.eye(3))
    with pytest.raises(ID11BError):
        batch.score_batch(np.eye(3)[None], gs, [0.1], tile=(3, 0))
    with pytest.raises(ID11BError):
        batch.score_batch(np.eye(3)[None], gs, [0.1], tile=(4, -1))


@pytest.mark.gpu
def test_refine_tuner(tune, oracle, cuda):
    from imaged11_b200 import batch, synth
    rng = np.random.default_rng(53)
    ng = 80
    counts = np.exp(rng.uniform(np.log(20), np.log(1500), ng)).astype(int)
    ps = synth.simulate(ng, "Ti_hcp", gmax=2.2, seed=54, noise_frac=0.0,
                        per_grain_counts=counts)
    idx, off = ps.grain_offsets()
    gv = ps.gv[idx]
    u0 = synth.perturb_ubis(ps.ubis, 0.2, 0.002, rng)
    gs = batch.GrainSet(gv, off, u0)
    best, table = tune.tune_refine(gs, 0.05, 3, reps=1)
    assert best in (32, 64, 128, 256) and gs.threads == best
    assert np.array_equal(gs.ubis.cpu().numpy().reshape(-1, 3, 3), u0)   # restored
    assert batch.GrainSet(gv, off, u0).threads == best                   # cached
    u, npk, _ = gs.refine(0.05, 3)
    ref_u, ref_n, _ = oracle.refine_csr(u0, gv, off, 0.05, 3)
    assert np.array_equal(npk.cpu().numpy(), ref_n)
    scale = np.abs(ref_u).reshape(ng, -1).max(1)
    err = np.abs(u.cpu().numpy() - ref_u).reshape(ng, -1).max(1)
    assert np.all(err <= 1e-11 * scale)


@pytest.mark.gpu
def test_grid_tuner(tune, oracle, cuda):
    from imaged11_b200 import batch, synth
    ps = synth.simulate(60, "Al", gmax=1.2, seed=55, noise_frac=0.1)
    rng = np.random.default_rng(56)
    ubis = synth.trial_ubis(ps.ubis, 500, 0.1, 0.5, rng)
    tols = [0.05, 0.1]
    best, table = tune.tune_grid(ubis, ps.gv, tols, reps=1)
    assert best in [t[:2] for t, _ in table]
    fastest = min(table, key=lambda x: x[1])[0]
    assert {t[2] for t, _ in table} == {"bins", "walk"}  # both methods timed
    assert tune.grid_method(len(ps.gv)) == fastest[2]
    grid = batch.GvecGrid(ps.gv)                      # picks the tuned shape
    assert grid.xsub == best[1]
    ref = oracle.score_many(ubis, ps.gv, tols)
    assert np.array_equal(batch.score_grid(ubis, grid, tols).cpu().numpy(), ref)
