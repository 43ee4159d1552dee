"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle.

Two libraries, both built by ``oracle/Makefile``:

* ``liboracle.so`` -- the C restatement of ImageD11's grain-scoring path
  (``oracle/id11_oracle.c``; each function cites the reference file:line it
  restates);
* ``_ref/libimaged11_ref.so`` -- the reference's own C sources
  (``src/closest.c``, ``src/cdiffraction.c``, ``src/cimaged11utils.c``)
  compiled unmodified, with OpenMP batch drivers (``oracle/ref_driver.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product (``imaged11_b200``) never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libimaged11_ref.so")

_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_p = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_p)


def _c64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


class _Lib:
    """Common wrapper: both libraries export the reference's function set,
    the oracle under an ``orc_`` prefix, the reference under its own names."""

    def __init__(self, path, prefix):
        self.path = path
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        L = self.lib
        f = self._f
        f("compute_gv").argtypes = [_p, _p, _d, _d, _d, _d, _p, _p, self._nt]
        f("compute_xlylzl").argtypes = [_p, _p, _p, _p, _p, _p, self._nt]
        f("compute_geometry").argtypes = [_p, _p, _d, _d, _d, _d, _p, _p, self._nt]
        f("score").argtypes = [_p, _p, _d, self._nt]
        f("score").restype = _i
        f("score_and_refine").argtypes = [_p, _p, _d, _p, _p, self._nt]
        f("refine_assigned").argtypes = [_p, _p, _p, _i, _p, _p, self._nt]
        f("score_and_assign").argtypes = [_p, _p, _d, _p, _p, _i, self._nt]
        f("score_and_assign").restype = _i
        f("verify_rounding").argtypes = [_i]
        f("verify_rounding").restype = _i
        del L

    @property
    def _nt(self):
        return _i64 if self.prefix else _i

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    # --- reference-shaped calls (numpy in, numpy out) ---
    def compute_gv(self, xlylzl, omega, omegasign, wvln, wedge, chi, t):
        x = _c64(xlylzl).reshape(-1, 3)
        om = _c64(omega)
        tt = _c64(t)
        gv = np.zeros_like(x)
        self._f("compute_gv")(_ptr(x), _ptr(om), omegasign, wvln, wedge, chi,
                              _ptr(tt), _ptr(gv), len(x))
        return gv

    def compute_geometry(self, xlylzl, omega, omegasign, wvln, wedge, chi, t):
        x = _c64(xlylzl).reshape(-1, 3)
        om = _c64(omega)
        tt = _c64(t)
        out = np.zeros((len(x), 6))
        self._f("compute_geometry")(_ptr(x), _ptr(om), omegasign, wvln, wedge,
                                    chi, _ptr(tt), _ptr(out), len(x))
        return out

    def compute_xlylzl(self, s, f, p, r, dist):
        s = _c64(s)
        f = _c64(f)
        p = _c64(p)
        r = _c64(r).ravel()
        dist = _c64(dist)
        out = np.zeros((len(s), 3))
        self._f("compute_xlylzl")(_ptr(s), _ptr(f), _ptr(p), _ptr(r), _ptr(dist),
                                  _ptr(out), len(s))
        return out

    def score(self, ubi, gv, tol):
        u = _c64(ubi, (3, 3))
        g = _c64(gv).reshape(-1, 3)
        return int(self._f("score")(_ptr(u), _ptr(g), tol, len(g)))

    def score_and_refine(self, ubi, gv, tol):
        """Returns (n, mean drlv2, refined ubi) -- ubi is not modified."""
        u = _c64(ubi, (3, 3)).copy()
        g = _c64(gv).reshape(-1, 3)
        n = ctypes.c_int(0)
        d = ctypes.c_double(0)
        self._f("score_and_refine")(_ptr(u), _ptr(g), tol, ctypes.byref(n),
                                    ctypes.byref(d), len(g))
        return n.value, d.value, u

    def refine_assigned(self, ubi, gv, labels, label):
        u = _c64(ubi, (3, 3)).copy()
        g = _c64(gv).reshape(-1, 3)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        n = ctypes.c_int(0)
        d = ctypes.c_double(0)
        self._f("refine_assigned")(_ptr(u), _ptr(g), _ptr(lab), int(label),
                                   ctypes.byref(n), ctypes.byref(d), len(g))
        return n.value, d.value, u

    def score_and_assign(self, ubi, gv, tol, drlv2, labels, label):
        """Returns (n, drlv2', labels') -- inputs are not modified."""
        u = _c64(ubi, (3, 3))
        g = _c64(gv).reshape(-1, 3)
        d = _c64(drlv2).copy()
        lab = np.ascontiguousarray(labels, dtype=np.int32).copy()
        n = self._f("score_and_assign")(_ptr(u), _ptr(g), tol, _ptr(d), _ptr(lab),
                                        int(label), len(g))
        return int(n), d, lab

    def verify_rounding(self, n):
        return int(self._f("verify_rounding")(n))


class Oracle(_Lib):
    """The C restatement (liboracle.so)."""

    def __init__(self, path=ORACLE_SO):
        super().__init__(path, "orc_")
        L = self.lib
        L.orc_score_many.argtypes = [_p, _i64, _p, _i64, _p, _i, _p]
        L.orc_refine_csr.argtypes = [_p, _p, _p, _i64, _d, _i, _p, _p]
        L.orc_inverse3x3.argtypes = [_p]
        L.orc_inverse3x3.restype = _i
        L.orc_wedgechi_matrix.argtypes = [_d, _d, _p]
        L.orc_max_threads.restype = _i

    def score_many(self, ubis, gv, tols):
        u = _c64(ubis).reshape(-1, 9)
        g = _c64(gv).reshape(-1, 3)
        t = _c64(np.atleast_1d(tols))
        out = np.zeros((len(u), len(t)), np.int32)
        self.lib.orc_score_many(_ptr(u), len(u), _ptr(g), len(g), _ptr(t), len(t),
                                _ptr(out))
        return out

    def refine_csr(self, ubis, gv, offsets, tol, iters):
        u = _c64(ubis).reshape(-1, 9).copy()
        g = _c64(gv).reshape(-1, 3)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        ng = len(off) - 1
        npk = np.zeros(ng, np.int32)
        d = np.zeros(ng)
        self.lib.orc_refine_csr(_ptr(u), _ptr(g), _ptr(off), ng, tol, iters,
                                _ptr(npk), _ptr(d))
        return u.reshape(-1, 3, 3), npk, d

    def inverse3x3(self, m):
        a = _c64(m).reshape(9).copy()
        rc = self.lib.orc_inverse3x3(_ptr(a))
        return rc, a.reshape(3, 3)

    def wedgechi_matrix(self, wedge, chi):
        m = np.zeros(9)
        self.lib.orc_wedgechi_matrix(wedge, chi, _ptr(m))
        return m.reshape(3, 3)

    def max_threads(self):
        return int(self.lib.orc_max_threads())


class Reference(_Lib):
    """The reference's own compiled C (oracle/_ref/libimaged11_ref.so)."""

    def __init__(self, path=REF_SO):
        super().__init__(path, "")
        L = self.lib
        L.ref_score_many.argtypes = [_p, _i64, _p, _i64, _p, _i, _p]
        L.ref_refine_csr.argtypes = [_p, _p, _p, _i64, _d, _i, _p, _p]
        L.ref_assign_seq.argtypes = [_p, _i64, _p, _i64, _d, _p, _p]
        L.ref_max_threads.restype = _i
        L.cimaged11_omp_set_num_threads.argtypes = [_i]

    def score_many(self, ubis, gv, tols):
        u = _c64(ubis).reshape(-1, 9)
        g = _c64(gv).reshape(-1, 3)
        t = _c64(np.atleast_1d(tols))
        out = np.zeros((len(u), len(t)), np.int32)
        self.lib.ref_score_many(_ptr(u), len(u), _ptr(g), len(g), _ptr(t), len(t),
                                _ptr(out))
        return out

    def refine_csr(self, ubis, gv, offsets, tol, iters):
        u = _c64(ubis).reshape(-1, 9).copy()
        g = _c64(gv).reshape(-1, 3)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        ng = len(off) - 1
        npk = np.zeros(ng, np.int32)
        d = np.zeros(ng)
        self.lib.ref_refine_csr(_ptr(u), _ptr(g), _ptr(off), ng, tol, iters,
                                _ptr(npk), _ptr(d))
        return u.reshape(-1, 3, 3), npk, d

    def assign_seq(self, ubis, gv, tol, drlv2, labels):
        """score_and_assign of grains 0 .. m-1 in order on (drlv2, labels),
        updated in place (float64 / int32 C arrays)."""
        u = _c64(ubis).reshape(-1, 9)
        g = _c64(gv).reshape(-1, 3)
        assert drlv2.dtype == np.float64 and labels.dtype == np.int32
        assert drlv2.flags.c_contiguous and labels.flags.c_contiguous
        self.lib.ref_assign_seq(_ptr(u), len(u), _ptr(g), len(g), float(tol), _ptr(drlv2),
                                _ptr(labels))

    def max_threads(self):
        return int(self.lib.ref_max_threads())


def build(ref_root=None):
    """Compile liboracle.so, and the reference library when its sources exist
    (ref_root, else the IMAGED11_REF environment variable: the root of an
    ImageD11 checkout; with neither, only the restatement is built)."""
    import subprocess
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    ref_root = ref_root or os.environ.get("IMAGED11_REF", "")
    subprocess.run(["make", "-s", "-C", HERE, "CC=" + cc, "REF=" + ref_root],
                   check=True)


def have_reference():
    return os.path.exists(REF_SO)
