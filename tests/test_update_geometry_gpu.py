"""Fused detector -> lab -> geometry pass (Ctransform.sf2geometry) against the
two separate drop-in calls (bit for bit) and against the oracle's
compute_xlylzl + compute_geometry (xyz bit for bit; angles and g within the
sin/cos tolerance of the other geometry tests)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GV_ULPS = 64


def _close_ulps(a, b, ulps):
    scale = np.abs(b).max(axis=-1, keepdims=True)
    return np.all(np.abs(a - b) <= ulps * np.spacing(scale))


def _pars(rng, tilt=True):
    return {"y_center": 1024.3, "z_center": 1021.7, "y_size": 75.0, "z_size": 75.2,
            "distance": 152300.0, "wavelength": 0.2846, "omegasign": -1.0,
            "tilt_x": 0.004 if tilt else 0.0, "tilt_y": -0.002 if tilt else 0.0,
            "tilt_z": 0.006 if tilt else 0.0, "o11": 1, "o12": 0, "o21": 0, "o22": -1,
            "wedge": 0.01 if tilt else 0.0, "chi": 0.02 if tilt else 0.0}


@pytest.mark.parametrize("tilt,t", [(True, (5.0, -3.0, 2.0)), (False, (0.0, 0.0, 0.0))])
def test_sf2geometry(oracle, tilt, t, cuda):
    import torch
    from imaged11_b200 import transform
    rng = np.random.default_rng(71)
    n = 100_003                                 # ragged final tile
    sc = rng.uniform(0, 2048, n)
    fc = rng.uniform(0, 2048, n)
    om = rng.uniform(-180, 360, n)
    sc[:3] = [1021.7, np.nan, 0.0]              # on the beam centre row, NaN, edge
    ct = transform.Ctransform(_pars(rng, tilt))
    xyz, out = ct.sf2geometry(sc, fc, om, *t)
    xyz2 = ct.sf2xyz(sc, fc)
    out2 = ct.xyz2geometry(xyz2, om, *t)
    assert np.array_equal(xyz, xyz2, equal_nan=True)
    assert np.array_equal(out, out2, equal_nan=True)
    ref_x = oracle.compute_xlylzl(sc, fc, ct.cen, ct.rmat, ct.distance_vec)
    assert np.array_equal(xyz, ref_x, equal_nan=True)
    p = ct.pars
    ref = oracle.compute_geometry(ref_x, om, p["omegasign"], p["wavelength"], p["wedge"],
                                  p["chi"], np.array(t))
    fin = np.isfinite(ref).all(1)
    assert np.array_equal(np.isfinite(out).all(1), fin)
    assert np.abs(out[fin, :2] - ref[fin, :2]).max() < 1e-11
    assert _close_ulps(out[fin, 3:], ref[fin, 3:], GV_ULPS)
    assert np.allclose(out[fin, 2], ref[fin, 2], rtol=1e-14, atol=0)
    # device tensors in, device tensors out, without the lab positions
    xd, od = ct.sf2geometry(torch.tensor(sc, device=cuda), torch.tensor(fc, device=cuda),
                            torch.tensor(om, device=cuda), *t, xyz=False)
    assert xd is None and od.is_cuda
    assert np.array_equal(od.cpu().numpy(), out, equal_nan=True)


def test_ctransform_methods_match_drop_in(cuda):
    from imaged11_b200 import transform
    rng = np.random.default_rng(72)
    ct = transform.Ctransform(_pars(rng))
    sc, fc, om = rng.uniform(0, 2048, 999), rng.uniform(0, 2048, 999), rng.uniform(0, 360, 999)
    g = ct.sf2gv(sc, fc, om, 1.0, 2.0, 3.0)
    out = ct.xyz2geometry(ct.sf2xyz(sc, fc), om, 1.0, 2.0, 3.0)
    assert np.array_equal(g, out[:, 3:])
    with pytest.raises(ValueError):
        ct.sf2geometry(sc, fc[:10], om)
