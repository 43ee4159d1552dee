"""Drop-in for the grain-scoring functions of ``ImageD11.cImageD11``.

Same names, positional/keyword arguments, return values, in-place outputs and
error behaviour as the reference's f2py module (``src/_cImageD11.pyf``), with
the work done by CUDA kernels on the current GPU:

=====================  ===============================================  ==========================
function               reference                                        returns
=====================  ===============================================  ==========================
compute_gv             src/cdiffraction.c:112-168, pyf:551-564          None (gv written)
compute_geometry       src/cdiffraction.c:31-94,   pyf:534-549          None (out written)
compute_xlylzl         src/cdiffraction.c:190-224, pyf:566-583          None (xlylzl written)
score                  src/closest.c:227-248,      pyf:106-120          int
score_and_refine       src/closest.c:267-345,      pyf:123-136          (n, mean drlv2); ubi refined
refine_assigned        src/closest.c:416-474,      pyf:156-170          (npk, mean drlv2); ubi refined
score_and_assign       src/closest.c:366-397,      pyf:138-154          int; drlv2, labels updated
verify_rounding        src/closest.c:100-119,      pyf:69-74            int (0 = good)
=====================  ===============================================  ==========================

Arrays may be numpy arrays (host; each call copies to the GPU and back through
the reference-signature C entry points) or CUDA ``torch.Tensor`` objects
(device; no copies, work enqueued on the current stream).

f2py conventions kept:

* ``intent(in)`` arrays are converted to C-contiguous float64 / int32 as
  needed (a copy, like f2py's silent cast);
* ``intent(inout)`` arrays (``gv`` of compute_gv, ``ubi`` of
  score_and_refine, ``drlv2``/``labels`` of score_and_assign, ...) must
  already be C-contiguous with the right element size, else ``ValueError``
  with f2py's message;
* ``refine_assigned``'s ``ubi`` is ``intent(c,in)`` but written by the C: the
  caller's array is refined in place only when it is C-contiguous float64,
  otherwise a converted copy is refined and the caller's array is unchanged;
* a singular least-squares system leaves the UBI unchanged (no error);
* ``score``, ``compute_gv`` and ``score_and_assign`` are not thread-safe in
  the reference; here every entry point may be called from several threads.
"""
import numpy as np

from . import _lib
from ._lib import lib, check, check_last

__all__ = [
    "compute_gv", "compute_geometry", "compute_xlylzl", "score", "score_and_refine",
    "refine_assigned", "score_and_assign", "verify_rounding",
    "cimaged11_omp_set_num_threads", "cimaged11_omp_get_max_threads",
    "cores_available", "OPENMP",
]

# The GPU module has no OpenMP; the thread knobs exist so callers that set them
# keep working (ImageD11/cImageD11.py:109-115).
OPENMP = False


def cimaged11_omp_set_num_threads(n):
    """Accepted for compatibility; the GPU path has no OpenMP threads."""
    return None


def cimaged11_omp_get_max_threads():
    """0, as for a reference build without OpenMP."""
    return 0


def cores_available():
    """Number of CPU cores usable by this process (ImageD11/cImageD11.py:89-106)."""
    import os
    if hasattr(os, "sched_getaffinity"):
        return max(1, len(os.sched_getaffinity(0)))
    return max(1, os.cpu_count() or 1)


# ---------------------------------------------------------------- helpers ----

def _torch():
    import torch
    return torch


def _is_cuda(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _ptr(a):
    return a.ctypes.data


def _in_f64(a, name, shape=None):
    """intent(in) float64: convert/copy like f2py."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        if a.size != int(np.prod(shape)) or (a.ndim > 1 and a.shape != tuple(shape)
                                             and len(shape) == a.ndim):
            raise ValueError("%s: expected shape %s, got %s" % (name, shape, a.shape))
        a = a.reshape(shape)
    return a


def _gv_in(gv, name="gv"):
    g = np.ascontiguousarray(gv, dtype=np.float64)
    if g.ndim != 2 or g.shape[1] != 3:
        raise ValueError("%s: 1-th dimension must be fixed to 3 but got %s" % (
            name, g.shape[1] if g.ndim == 2 else g.shape))
    return g


def _inout(a, dtype, name, shape=None):
    """intent(inout): must be C-contiguous with the right element size."""
    if not isinstance(a, np.ndarray):
        raise ValueError("failed to initialize intent(inout) array -- expected an array")
    if a.dtype.itemsize != np.dtype(dtype).itemsize:
        raise ValueError("failed to initialize intent(inout) array -- expected elsize=%d "
                         "but got %d" % (np.dtype(dtype).itemsize, a.dtype.itemsize))
    if not a.flags.c_contiguous:
        raise ValueError("failed to initialize intent(inout) array -- input not contiguous")
    if a.dtype != np.dtype(dtype):
        raise ValueError("failed to initialize intent(inout) array -- expected %s but got %s"
                         % (np.dtype(dtype), a.dtype))
    if shape is not None and a.shape != tuple(shape):
        raise ValueError("%s: expected shape %s, got %s" % (name, tuple(shape), a.shape))
    return a


def _dev_f64(t, name, cols=None):
    torch = _torch()
    if t.dtype != torch.float64:
        raise ValueError("%s: CUDA tensor must be float64" % name)
    if not t.is_contiguous():
        raise ValueError("%s: CUDA tensor must be contiguous" % name)
    if cols is not None and (t.dim() != 2 or t.shape[1] != cols):
        raise ValueError("%s: expected shape (n, %d), got %s" % (name, cols, tuple(t.shape)))
    return t


def _stream():
    return _torch().cuda.current_stream().cuda_stream


def _to_dev(a, dtype=None):
    torch = _torch()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype), device="cuda")


# -------------------------------------------------------------- geometry ----

def compute_gv(xlylzl, omega, omegasign, wvln, wedge, chi, t, gv):
    """compute_gv computes scattering vectors given the positions of the spot in
    the laboratory in xlylzl[npks], the omega rotation[npks], and the rest of
    the parameters (wedge, wvln, chi, t[3] and omegasign).  gv (npks,3) is
    written in place."""
    tt = np.ascontiguousarray(t, dtype=np.float64).reshape(3)
    if _is_cuda(gv) or _is_cuda(xlylzl):
        x = _dev_f64(xlylzl, "xlylzl", 3)
        om = _dev_f64(omega, "omega")
        g = _dev_f64(gv, "gv", 3)
        if x.shape[0] != om.shape[0] or g.shape[0] != x.shape[0]:
            raise ValueError("compute_gv: xlylzl, omega and gv lengths differ")
        check(lib.id11b_dev_compute_gv(x.data_ptr(), om.data_ptr(), omegasign, wvln, wedge,
                                       chi, _ptr(tt), g.data_ptr(), None, x.shape[0],
                                       _stream()), "compute_gv")
        return None
    x = _gv_in(xlylzl, "xlylzl")
    om = np.ascontiguousarray(omega, dtype=np.float64).reshape(-1)
    n = x.shape[0]
    if om.shape[0] != n:
        raise ValueError("compute_gv: omega has %d values for %d peaks" % (om.shape[0], n))
    _inout(gv, np.float64, "gv", (n, 3))
    lib.id11b_compute_gv(_ptr(x), _ptr(om), float(omegasign), float(wvln), float(wedge),
                         float(chi), _ptr(tt), _ptr(gv), n)
    check_last("compute_gv")
    return None


def compute_geometry(xlylzl, omega, omegasign, wvln, wedge, chi, t, out):
    """compute_geometry computes tth, eta, ds, gx, gy, gz into out (npks,6)."""
    tt = np.ascontiguousarray(t, dtype=np.float64).reshape(3)
    if _is_cuda(out) or _is_cuda(xlylzl):
        x = _dev_f64(xlylzl, "xlylzl", 3)
        om = _dev_f64(omega, "omega")
        o = _dev_f64(out, "out", 6)
        if x.shape[0] != om.shape[0] or o.shape[0] != x.shape[0]:
            raise ValueError("compute_geometry: lengths differ")
        check(lib.id11b_dev_compute_geometry(x.data_ptr(), om.data_ptr(), omegasign, wvln,
                                             wedge, chi, _ptr(tt), o.data_ptr(), x.shape[0],
                                             _stream()), "compute_geometry")
        return None
    x = _gv_in(xlylzl, "xlylzl")
    om = np.ascontiguousarray(omega, dtype=np.float64).reshape(-1)
    n = x.shape[0]
    if om.shape[0] != n:
        raise ValueError("compute_geometry: omega has %d values for %d peaks" % (om.shape[0], n))
    _inout(out, np.float64, "out", (n, 6))
    lib.id11b_compute_geometry(_ptr(x), _ptr(om), float(omegasign), float(wvln), float(wedge),
                               float(chi), _ptr(tt), _ptr(out), n)
    check_last("compute_geometry")
    return None


def compute_xlylzl(s, f, p, r, dist, xlylzl):
    """compute_xlylzl finds spot positions in the laboratory frame.
    p = [s_cen, f_cen, s_size, f_size]; r[9] = detector_rotation_matrix .
    flipmatrix; dist = [distancex, distancey, distancez]."""
    pp = _in_f64(p, "p").reshape(4)
    rr = _in_f64(r, "r").reshape(9)
    dd = _in_f64(dist, "dist").reshape(3)
    if _is_cuda(xlylzl) or _is_cuda(s):
        sv = _dev_f64(s, "s")
        fv = _dev_f64(f, "f")
        x = _dev_f64(xlylzl, "xlylzl", 3)
        if sv.shape[0] != fv.shape[0] or x.shape[0] != sv.shape[0]:
            raise ValueError("compute_xlylzl: lengths differ")
        check(lib.id11b_dev_compute_xlylzl(sv.data_ptr(), fv.data_ptr(), _ptr(pp), _ptr(rr),
                                           _ptr(dd), x.data_ptr(), sv.shape[0], _stream()),
              "compute_xlylzl")
        return None
    sv = np.ascontiguousarray(s, dtype=np.float64).reshape(-1)
    fv = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
    n = sv.shape[0]
    if fv.shape[0] != n:
        raise ValueError("compute_xlylzl: s and f lengths differ")
    _inout(xlylzl, np.float64, "xlylzl", (n, 3))
    lib.id11b_compute_xlylzl(_ptr(sv), _ptr(fv), _ptr(pp), _ptr(rr), _ptr(dd), _ptr(xlylzl), n)
    check_last("compute_xlylzl")
    return None


# --------------------------------------------------------------- scoring ----

def _dev_ubi(ubi):
    """UBI as a (9,) float64 CUDA tensor; returns (tensor, is_callers_tensor)."""
    torch = _torch()
    if _is_cuda(ubi):
        if ubi.dtype != torch.float64 or not ubi.is_contiguous() or ubi.numel() != 9:
            raise ValueError("ubi: CUDA tensor must be contiguous float64 with 9 elements")
        return ubi.view(9), True
    return _to_dev(np.asarray(ubi, dtype=np.float64).reshape(9)), False


def score(ubi, gv, tol):
    """score takes a ubi matrix and list of g-vectors and computes
    hkl = dot(ubi, gv), then rounds these to integer and computes
    drlv2 = (h-int(h))**2 + (k-int(k))**2 + (l-int(l))**2.  If drlv2 is less
    than tol*tol then the peak is considered to be indexed.  Returns the number
    of peaks found."""
    if _is_cuda(gv):
        torch = _torch()
        g = _dev_f64(gv, "gv", 3)
        u, _ = _dev_ubi(ubi)
        c = torch.empty(1, dtype=torch.int32, device=g.device)
        check(lib.id11b_dev_score(u.data_ptr(), g.data_ptr(), float(tol), g.shape[0],
                                  c.data_ptr(), _stream()), "score")
        return int(c.item())
    u = _in_f64(ubi, "ubi", (3, 3))
    g = _gv_in(gv)
    n = lib.id11b_score(_ptr(u), _ptr(g), float(tol), g.shape[0])
    check_last("score")
    return int(n)


def _lsq_dev(mode, ubi, gv, tol, labels, label):
    torch = _torch()
    g = _dev_f64(gv, "gv", 3)
    u, own = _dev_ubi(ubi)
    ng = g.shape[0]
    wsb = lib.id11b_lsq_workspace_bytes(ng)
    ws = torch.empty(wsb, dtype=torch.uint8, device=g.device)
    n = torch.empty(1, dtype=torch.int32, device=g.device)
    m = torch.empty(1, dtype=torch.float64, device=g.device)
    if mode == 0:
        check(lib.id11b_dev_score_and_refine(u.data_ptr(), g.data_ptr(), float(tol), ng,
                                             n.data_ptr(), m.data_ptr(), ws.data_ptr(), wsb,
                                             _stream()), "score_and_refine")
    else:
        lab = labels if _is_cuda(labels) else _to_dev(labels, np.int32)
        if lab.dtype != torch.int32 or not lab.is_contiguous() or lab.numel() != ng:
            raise ValueError("labels: expected %d contiguous int32 values" % ng)
        check(lib.id11b_dev_refine_assigned(u.data_ptr(), g.data_ptr(), lab.data_ptr(),
                                            int(label), ng, n.data_ptr(), m.data_ptr(),
                                            ws.data_ptr(), wsb, _stream()), "refine_assigned")
    if not own and isinstance(ubi, np.ndarray) and ubi.flags.c_contiguous and \
            ubi.dtype == np.float64:
        ubi.reshape(9)[:] = u.cpu().numpy()
    return int(n.item()), float(m.item())


def score_and_refine(ubi, gv, tol):
    """score_and_refine is very similar to score but it also refines the UB
    matrix using the assigned peaks and overwrites the argument.  It returns the
    number of peaks and fit prior to refinement."""
    if _is_cuda(ubi):
        return _lsq_dev(0, ubi, gv, tol, None, 0)
    _inout(ubi, np.float64, "ubi", (3, 3))
    if _is_cuda(gv):
        return _lsq_dev(0, ubi, gv, tol, None, 0)
    g = _gv_in(gv)
    n = _lib.ctypes.c_int(0)
    d = _lib.ctypes.c_double(0.)
    lib.id11b_score_and_refine(_ptr(ubi), _ptr(g), float(tol), _lib.ctypes.addressof(n),
                               _lib.ctypes.addressof(d), g.shape[0])
    check_last("score_and_refine")
    return n.value, d.value


def refine_assigned(ubi, gv, labels, label):
    """refine_assigned fits a ubi matrix to a set of g-vectors and assignments
    in labels, i.e. where(labels==label) it uses the peaks.  Returns
    (npk, mean drlv2)."""
    if _is_cuda(ubi) or _is_cuda(gv):
        return _lsq_dev(1, ubi, gv, 0., labels, label)
    if isinstance(ubi, np.ndarray) and ubi.dtype == np.float64 and ubi.flags.c_contiguous \
            and ubi.size == 9:
        u = ubi                       # f2py passes the caller's buffer: refined in place
    else:
        u = _in_f64(ubi, "ubi", (3, 3)).copy()
    g = _gv_in(gv)
    lab = np.ascontiguousarray(labels, dtype=np.int32).reshape(-1)
    if lab.shape[0] != g.shape[0]:
        raise ValueError("refine_assigned: labels has %d values for %d g-vectors"
                         % (lab.shape[0], g.shape[0]))
    n = _lib.ctypes.c_int(0)
    d = _lib.ctypes.c_double(0.)
    lib.id11b_refine_assigned(_ptr(u), _ptr(g), _ptr(lab), int(label),
                              _lib.ctypes.addressof(n), _lib.ctypes.addressof(d), g.shape[0])
    check_last("refine_assigned")
    return n.value, d.value


def score_and_assign(ubi, gv, tol, drlv2, labels, label):
    """score_and_assign is similar to score but it assigns peaks to this ubi
    only if they fit the data better than the current UBI.  It updates drlv2
    and labels to use the best fitting grain for each peak."""
    if _is_cuda(gv):
        torch = _torch()
        g = _dev_f64(gv, "gv", 3)
        u, _ = _dev_ubi(ubi)
        ng = g.shape[0]
        if not (_is_cuda(drlv2) and _is_cuda(labels)):
            raise ValueError("score_and_assign: drlv2 and labels must be CUDA tensors "
                             "when gv is")
        if drlv2.dtype != torch.float64 or not drlv2.is_contiguous() or drlv2.numel() != ng:
            raise ValueError("failed to initialize intent(inout) array -- drlv2")
        if labels.dtype != torch.int32 or not labels.is_contiguous() or labels.numel() != ng:
            raise ValueError("failed to initialize intent(inout) array -- labels")
        c = torch.empty(1, dtype=torch.int32, device=g.device)
        check(lib.id11b_dev_score_and_assign(u.data_ptr(), g.data_ptr(), float(tol),
                                             drlv2.data_ptr(), labels.data_ptr(), int(label),
                                             ng, c.data_ptr(), _stream()), "score_and_assign")
        return int(c.item())
    u = _in_f64(ubi, "ubi", (3, 3))
    g = _gv_in(gv)
    ng = g.shape[0]
    _inout(drlv2, np.float64, "drlv2", (ng,))
    _inout(labels, np.int32, "labels", (ng,))
    n = lib.id11b_score_and_assign(_ptr(u), _ptr(g), float(tol), _ptr(drlv2), _ptr(labels),
                                   int(label), ng)
    check_last("score_and_assign")
    return int(n)


def verify_rounding(n):
    """Checks that the GPU's round-to-nearest-integer code is correct
    (0 = no mismatch)."""
    r = lib.id11b_verify_rounding(int(n))
    check_last("verify_rounding")
    return int(r)
