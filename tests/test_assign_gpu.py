"""Batched score_and_assign through the cell index vs the oracle's sequence
of score_and_assign calls (the loop of ImageD11/indexing.py fight_over_peaks).

Labels and drlv2 must match the sequential calls bit for bit: ties go to the
first grain, the reference's "does not belong after all" reset applies to g
that held a grain's label, and g outside the regular range follow the same
sequence of calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
METHODS = ["walk", "bins"]   # the lookup and the binned join


def sequential(oracle, ubis, gv, tol, drlv2, labels, grain_labels):
    d, lab = drlv2.copy(), labels.copy()
    for u, gl in zip(ubis, grain_labels):
        _, d, lab = oracle.score_and_assign(u, gv, tol, d, lab, int(gl))
    return d, lab


@pytest.fixture(scope="module")
def scene():
    from imaged11_b200 import synth
    ps = synth.simulate(150, "Al", gmax=1.3, seed=61, noise_frac=0.10)
    rng = np.random.default_rng(62)
    ubis = synth.trial_ubis(ps.ubis, 400, 0.5, 0.3, rng)
    return ps, ubis


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("tol", [0.02, 0.1, 0.3])
def test_fight_over_peaks(scene, oracle, tol, method, cuda):
    from imaged11_b200 import batch
    ps, ubis = scene
    n = len(ps.gv)
    d0 = np.zeros(n) + 2
    l0 = np.zeros(n, np.int32) - 1
    ref_d, ref_l = sequential(oracle, ubis, ps.gv, tol, d0, l0, range(len(ubis)))
    d, lab = d0.copy(), l0.copy()
    npk = batch.score_and_assign_grid(ubis, batch.GvecGrid(ps.gv), tol, d, lab, npk=True,
                                      method=method)
    assert np.array_equal(lab, ref_l)
    assert np.array_equal(d, ref_d)
    hist = np.bincount(ref_l[ref_l >= 0], minlength=len(ubis))
    assert np.array_equal(npk.cpu().numpy(), hist)


@pytest.mark.parametrize("method", METHODS)
def test_ties_labels_and_resets(scene, oracle, method, cuda):
    from imaged11_b200 import batch
    ps, ubis = scene
    u = ubis[:60].copy()
    u[7] = u[3]                       # exact ties: the first grain keeps the peak
    u[11] = 0.0                       # singular: plain scan
    u[13, 0, 0] = np.nan
    gl = np.arange(60, dtype=np.int32) * 10 + 5
    n = len(ps.gv)
    rng = np.random.default_rng(63)
    d0 = rng.uniform(0.0, 0.02, n)    # some peaks already well assigned
    d0[rng.random(n) < 0.05] = -1.0   # never reassigned
    l0 = rng.choice(np.concatenate([gl, [-1, 3, 99999]]), n).astype(np.int32)
    ref_d, ref_l = sequential(oracle, u, ps.gv, 0.08, d0, l0, gl)
    d, lab = d0.copy(), l0.copy()
    batch.score_and_assign_grid(u, batch.GvecGrid(ps.gv), 0.08, d, lab, grain_labels=gl,
                                method=method)
    assert np.array_equal(lab, ref_l)
    assert np.array_equal(d, ref_d)


def test_bins_workspace_ranges(scene, oracle, cuda):
    """The binned assignment with a workspace holding part of the boxes: the
    grains run in ranges, each range's boxes rebuilt for the second pass after
    the first pass has seen every range; too small for one grain's boxes is an
    error."""
    from imaged11_b200 import batch
    from imaged11_b200._lib import ID11BError
    ps, ubis = scene
    u = ubis[:120]
    n = len(ps.gv)
    d0 = np.zeros(n) + 2
    l0 = np.zeros(n, np.int32) - 1
    ref_d, ref_l = sequential(oracle, u, ps.gv, 0.1, d0, l0, range(len(u)))
    grid = batch.GvecGrid(ps.gv)
    est = batch.bins_box_estimate(u, grid, 0.1)
    for frac in (0.5, 0.13):
        ws = batch.BinsWorkspace(len(u), grid, int(est * frac))
        d, lab = d0.copy(), l0.copy()
        batch.score_and_assign_grid(u, grid, 0.1, d, lab, method="bins", workspace=ws)
        assert np.array_equal(lab, ref_l), frac
        assert np.array_equal(d, ref_d), frac
    with pytest.raises(ID11BError):
        batch.score_and_assign_grid(u, grid, 0.1, d0.copy(), l0.copy(), method="bins",
                                    workspace=batch.BinsWorkspace(len(u), grid, 10))


@pytest.mark.parametrize("method", METHODS)
def test_special_g_and_device_tensors(golden, oracle, method, cuda):
    import torch
    from imaged11_b200 import batch
    dd = golden["scoring"]
    gv = dd["adv_gv"]
    ubis = np.concatenate([dd["adv_ubi"][None], dd["sc_ubis"][:9]])
    n = len(gv)
    d0 = np.zeros(n) + 2
    l0 = np.zeros(n, np.int32) - 1
    ref_d, ref_l = sequential(oracle, ubis, gv, 0.1, d0, l0, range(len(ubis)))
    d = torch.tensor(d0, device="cuda")
    lab = torch.tensor(l0, device="cuda")
    batch.score_and_assign_grid(ubis, batch.GvecGrid(gv), 0.1, d, lab, method=method)
    assert np.array_equal(lab.cpu().numpy(), ref_l)
    assert np.array_equal(d.cpu().numpy(), ref_d, equal_nan=True)


def test_bad_grain_labels(scene, cuda):
    from imaged11_b200 import batch
    ps, ubis = scene
    n = len(ps.gv)
    d, lab = np.zeros(n) + 2, np.zeros(n, np.int32) - 1
    with pytest.raises(ValueError):
        batch.score_and_assign_grid(ubis[:3], batch.GvecGrid(ps.gv), 0.1, d, lab,
                                    grain_labels=[3, 2, 5])


def test_sharded_passes_on_one_gpu(scene, oracle, cuda):
    """The sharded driver with the CUDA passes (world 1 over gloo; the
    multi-rank exchange itself is covered by tests/test_multirank.py)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    from imaged11_b200 import batch, shard
    ps, ubis = scene
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        grid = batch.GvecGrid(ps.gv)
        n = len(ps.gv)
        d = torch.full((n,), 2.0, dtype=torch.float64, device=cuda)
        lab = torch.full((n,), -1, dtype=torch.int32, device=cuda)
        shard.score_and_assign_sharded(ubis, 0.1, d, lab, shard.CudaAssignPasses(grid),
                                       device="cpu")
        d2 = torch.full((n,), 2.0, dtype=torch.float64, device=cuda)
        lab2 = torch.full((n,), -1, dtype=torch.int32, device=cuda)
        batch.score_and_assign_grid(ubis, grid, 0.1, d2, lab2)
        assert torch.equal(lab, lab2) and torch.equal(d, d2)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("method", METHODS)
def test_random_sweep(oracle, method, cuda):
    from imaged11_b200 import batch
    rng = np.random.default_rng(79)
    for trial in range(10):
        n = int(rng.integers(1, 3000))
        gv = rng.normal(size=(n, 3)) * rng.uniform(0.3, 1.5)
        m = int(rng.integers(1, 60))
        ubis = np.empty((m, 3, 3))
        for i in range(m):
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            ubis[i] = np.diag(rng.uniform(2.0, 10.0, 3)) @ q.T
        ubis[m // 2] = ubis[0]                      # a tie
        tol = float(rng.uniform(0.01, 0.4))
        d0 = rng.uniform(0.0, 0.2, n)
        l0 = rng.choice(np.arange(-1, m + 3), n).astype(np.int32)
        d, lab = d0.copy(), l0.copy()
        for i, u in enumerate(ubis):
            _, d, lab = oracle.score_and_assign(u, gv, tol, d, lab, i)
        dd, ll = d0.copy(), l0.copy()
        batch.score_and_assign_grid(ubis, batch.GvecGrid(gv), tol, dd, ll, method=method)
        assert np.array_equal(ll, lab), trial
        assert np.array_equal(dd, d), trial
