"""Ctransform: the reference's detector-geometry helper (ImageD11/transform.py
:655-774) over this package's kernels, plus the fused update_geometry pass.

The parameter handling repeats the reference's numpy steps (same matrices,
same products) so that the r, p and dist handed to the kernels carry the same
bits as the reference's; the per-peak work runs on the GPU.  Arrays may be
numpy (results come back as numpy) or CUDA tensors (results stay on the GPU).
"""
import numpy as np

from . import cImageD11
from ._lib import lib, check


def _torch():
    import torch
    return torch


def detector_rotation_matrix(tilt_x, tilt_y, tilt_z):
    """R3(tilt_x).R2(tilt_y).R1(tilt_z), tilts in radians
    (ImageD11/transform.py:51-82)."""
    r1 = np.array([[np.cos(tilt_z), -np.sin(tilt_z), 0],
                   [np.sin(tilt_z), np.cos(tilt_z), 0],
                   [0, 0, 1]], float)
    r2 = np.array([[np.cos(tilt_y), 0, np.sin(tilt_y)],
                   [0, 1, 0],
                   [-np.sin(tilt_y), 0, np.cos(tilt_y)]], float)
    r3 = np.array([[1, 0, 0],
                   [0, np.cos(tilt_x), -np.sin(tilt_x)],
                   [0, np.sin(tilt_x), np.cos(tilt_x)]], float)
    return np.dot(np.dot(r3, r2), r1)


class Ctransform(object):
    """Same constructor and methods as ImageD11.transform.Ctransform."""

    pnames = ("y_center", "z_center", "y_size", "z_size", "distance", "wavelength",
              "omegasign", "tilt_x", "tilt_y", "tilt_z", "o11", "o12", "o21", "o22",
              "wedge", "chi")

    def __init__(self, pars):
        self.pars = {}
        for p in self.pnames:
            self.pars[p] = pars[p]
        self.reset()

    def reset(self):
        p = self.pars
        self.distance_vec = np.array((p["distance"], 0.0, 0.0))
        self.dmat = detector_rotation_matrix(p["tilt_x"], p["tilt_y"], p["tilt_z"])
        self.fmat = np.array([[1, 0, 0], [0, p["o22"], p["o21"]], [0, p["o12"], p["o11"]]])
        self.rmat = np.dot(self.dmat, self.fmat).ravel()
        self.cen = np.array((p["z_center"], p["y_center"], p["z_size"], p["y_size"]))

    # -- the reference's methods ------------------------------------------
    def sf2xyz(self, sc, fc, out=None):
        if len(sc) != len(fc):
            raise ValueError("sc and fc lengths differ")
        if out is None:
            out = self._empty(sc, (len(sc), 3))
        cImageD11.compute_xlylzl(sc, fc, self.cen, self.rmat, self.distance_vec, out)
        return out

    def xyz2gv(self, xyz, omega, tx=0, ty=0, tz=0, out=None):
        if len(omega) != len(xyz):
            raise ValueError("xyz and omega lengths differ")
        if out is None:
            out = self._empty(xyz, (len(xyz), 3))
        p = self.pars
        cImageD11.compute_gv(xyz, omega, p["omegasign"], p["wavelength"], p["wedge"],
                             p["chi"], np.array((tx, ty, tz)), out)
        return out

    def sf2gv(self, sc, fc, omega, tx=0, ty=0, tz=0, out=None):
        return self.xyz2gv(self.sf2xyz(sc, fc), omega, tx, ty, tz, out)

    def xyz2geometry(self, xyz, omega, tx=0, ty=0, tz=0, out=None):
        if len(omega) != len(xyz) or xyz.shape[1] != 3:
            raise ValueError("xyz must be (n,3) with one omega per row")
        if out is None:
            out = self._empty(xyz, (len(xyz), 6))
        p = self.pars
        cImageD11.compute_geometry(xyz, omega, p["omegasign"], p["wavelength"], p["wedge"],
                                   p["chi"], np.array((tx, ty, tz)), out)
        return out

    # -- fused ---------------------------------------------------------------
    def sf2geometry(self, sc, fc, omega, tx=0, ty=0, tz=0, xyz=True):
        """sf2xyz then xyz2geometry in one GPU pass (what updateGeometry's fast
        path does in two, ImageD11/columnfile.py:497-504).  Returns
        (xyz (n,3) or None, out (n,6) = tth, eta, ds, gx, gy, gz), identical to
        the two calls."""
        torch = _torch()
        host = not (torch.is_tensor(sc) and sc.is_cuda)
        dev = torch.device("cuda", torch.cuda.current_device()) if host else sc.device

        def d(a):
            if torch.is_tensor(a):
                return a.to(dev, torch.float64).contiguous().reshape(-1)
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(-1),
                                   device=dev)
        s, f, om = d(sc), d(fc), d(omega)
        n = s.numel()
        if f.numel() != n or om.numel() != n:
            raise ValueError("sc, fc and omega lengths differ")
        out = torch.empty((n, 6), dtype=torch.float64, device=dev)
        x = torch.empty((n, 3), dtype=torch.float64, device=dev) if xyz else None
        p = self.pars
        cen = np.ascontiguousarray(self.cen, dtype=np.float64)
        rm = np.ascontiguousarray(self.rmat, dtype=np.float64)
        dv = np.ascontiguousarray(self.distance_vec, dtype=np.float64)
        t = np.array((tx, ty, tz), dtype=np.float64)
        check(lib.id11b_dev_update_geometry(s.data_ptr(), f.data_ptr(), om.data_ptr(),
                                            cen.ctypes.data, rm.ctypes.data, dv.ctypes.data,
                                            float(p["omegasign"]), float(p["wavelength"]),
                                            float(p["wedge"]), float(p["chi"]), t.ctypes.data,
                                            x.data_ptr() if xyz else None, out.data_ptr(),
                                            None, n, torch.cuda.current_stream().cuda_stream),
              "update_geometry")
        if host:
            return (x.cpu().numpy() if xyz else None), out.cpu().numpy()
        return x, out

    @staticmethod
    def _empty(like, shape):
        torch = _torch()
        if torch.is_tensor(like) and like.is_cuda:
            return torch.empty(shape, dtype=torch.float64, device=like.device)
        return np.empty(shape, float)
