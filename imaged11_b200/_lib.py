"""ctypes binding of libimaged11_b200.so (the C ABI in include/imaged11_b200.h).

The library is required: importing this module without it, or calling a
device entry point on a machine without a CUDA device, raises.  There is no
CPU fallback anywhere in the package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# IMAGED11_B200_LIB may name another build of the same library (e.g. one
# compiled with different tuning constants); default: the in-tree build.
LIB_PATH = os.environ.get("IMAGED11_B200_LIB") or os.path.join(HERE, "libimaged11_b200.so")

_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_p = ctypes.c_void_p

# (name, restype, argtypes) for every exported entry point
_SIGNATURES = [
    ("id11b_version", _i, []),
    ("id11b_status_string", ctypes.c_char_p, [_i]),
    ("id11b_last_cuda_error", _i, []),
    ("id11b_last_status", _i, []),
    # layer 1: reference signatures, host pointers
    ("id11b_compute_gv", None, [_p, _p, _d, _d, _d, _d, _p, _p, _i]),
    ("id11b_compute_geometry", None, [_p, _p, _d, _d, _d, _d, _p, _p, _i]),
    ("id11b_compute_xlylzl", None, [_p, _p, _p, _p, _p, _p, _i]),
    ("id11b_score", _i, [_p, _p, _d, _i]),
    ("id11b_score_and_refine", None, [_p, _p, _d, _p, _p, _i]),
    ("id11b_refine_assigned", None, [_p, _p, _p, _i, _p, _p, _i]),
    ("id11b_score_and_assign", _i, [_p, _p, _d, _p, _p, _i, _i]),
    ("id11b_verify_rounding", _i, [_i]),
    # layer 2: device pointers + stream
    ("id11b_dev_compute_gv", _i, [_p, _p, _d, _d, _d, _d, _p, _p, _p, _i64, _p]),
    ("id11b_dev_compute_geometry", _i, [_p, _p, _d, _d, _d, _d, _p, _p, _i64, _p]),
    ("id11b_dev_compute_xlylzl", _i, [_p, _p, _p, _p, _p, _p, _i64, _p]),
    ("id11b_dev_update_geometry", _i, [_p, _p, _p, _p, _p, _p, _d, _d, _d, _d, _p, _p, _p, _p,
                                        _i64, _p]),
    ("id11b_dev_score", _i, [_p, _p, _d, _i64, _p, _p]),
    ("id11b_lsq_workspace_bytes", _i64, [_i64]),
    ("id11b_dev_score_and_refine", _i, [_p, _p, _d, _i64, _p, _p, _p, _i64, _p]),
    ("id11b_dev_refine_assigned", _i, [_p, _p, _p, _i, _i64, _p, _p, _p, _i64, _p]),
    ("id11b_noalloc_scratch_bytes", _i64, []),
    ("id11b_dev_score_and_refine_noalloc", _i, [_p, _p, _d, _i64, _p, _p, _p]),
    ("id11b_dev_score_and_assign", _i, [_p, _p, _d, _p, _p, _i, _i64, _p, _p]),
    ("id11b_dev_verify_rounding", _i, [_i, _p, _p]),
    ("id11b_dev_score_many_fp64", _i, [_p, _i64, _p, _i64, _p, _i, _p, _p]),
    ("id11b_gvec_workspace_bytes", _i64, [_i64]),
    ("id11b_dev_prepare_gvecs", _i, [_p, _i64, _p, _p, _i64, _p]),
    ("id11b_batch_workspace_bytes", _i64, [_i64, _i64, _i]),
    ("id11b_dev_score_batch", _i, [_p, _i64, _p, _p, _i64, _p, _p, _i, _p, _p, _p, _i64, _p]),
    ("id11b_score_tile_default", _i, [_i64, _i64, _p, _p]),
    ("id11b_dev_score_batch_tiled", _i, [_p, _i64, _p, _p, _i64, _p, _p, _i, _p, _p, _i, _i,
                                          _p, _i64, _p]),
    ("id11b_dev_gvec_bounds", _i, [_p, _i64, _p, _p]),
    ("id11b_grid_plan", _i, [ctypes.c_float, _i64, _d, _p, _p]),
    ("id11b_grid_bytes", _i64, [_i64, _i, _i]),
    ("id11b_dev_build_grid", _i, [_p, _i64, ctypes.c_float, ctypes.c_float, _d, _i, _i, _p,
                                   _i64, _p]),
    ("id11b_grid_score_workspace_bytes", _i64, [_i64, _i]),
    ("id11b_dev_score_grid", _i, [_p, _i64, _p, _i64, _i, _i, _p, _p, _i, _p, _p, _p, _i64,
                                   _p]),
    ("id11b_grid_stats", _i, [_p, _p, _p, _p, _p, _p, _p]),
    ("id11b_grid_bins_time_join", _i, [_p, _p]),
    ("id11b_grid_bins_workspace_bytes", _i64, [_i64, _i, _i, _i64]),
    ("id11b_dev_score_grid_bins", _i, [_p, _i64, _p, _i64, _i, _i, _p, _p, _i, _p, _p, _p,
                                        _i64, _p]),
    ("id11b_grid_refine_workspace_bytes", _i64, [_i64]),
    ("id11b_dev_refine_grid", _i, [_p, _i64, _p, _i64, _i, _i, _p, _d, _i, _p, _p, _p, _i64,
                                    _p]),
    ("id11b_assign_workspace_bytes", _i64, [_i64]),
    ("id11b_dev_assign_grid_pass", _i, [_p, _i64, _i64, _i64, _i, _i, _p, _d, _p, _i, _p, _p,
                                         _p]),
    ("id11b_dev_assign_grid_bins", _i, [_p, _i64, _p, _i64, _i, _i, _p, _d, _p, _p, _p, _p, _i64,
                                        _p]),
    ("id11b_dev_assign_grid_final", _i, [_p, _i64, _p, _p, _i64, _i, _i, _p, _d, _p, _p, _p, _p,
                                          _p, _p]),
    ("id11b_dev_score_and_assign_grid", _i, [_p, _i64, _p, _p, _i64, _i, _i, _p, _d, _p, _p,
                                              _p, _p, _i64, _p]),
    ("id11b_dev_refine_batch", _i, [_p, _i64, _p, _p, _i64, _p, _d, _i, _p, _p, _p, _i64, _p]),
    ("id11b_batch_stats", _i, [_p, _i64, _i64, _i, _p, _p, _p, _p]),
    ("id11b_refine_csr_workspace_bytes", _i64, []),
    ("id11b_dev_refine_csr", _i, [_p, _p, _p, _p, _i, _d, _i, _i, _i, _p, _p, _p, _i64, _p]),
    ("id11b_dev_refine_csr_f32c", _i, [_p, _p, _p, _p, _i, _d, _i, _d, _p, _p, _p, _i64, _p]),
    ("id11b_dev_refine_translations", _i, [_p, _p, _p, _i, _p, _p, _d, _d, _d, _d, _d, _i, _p,
                                            _p, _p, _p]),
    ("id11b_adjoint_workspace_bytes", _i64, [_i]),
    ("id11b_dev_residuals", _i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p, _p]),
    ("id11b_dev_residuals_adjoint", _i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p,
                                          _p, _i64, _p]),
    ("id11b_dev_residual_loss", _i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p, _p,
                                      _p, _i64, _p]),
    ("id11b_dev_best_ubis", _i, [_p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p]),
    ("id11b_dev_omega_sincos", _i, [_p, _i64, _d, _p, _p]),
    ("id11b_dev_bragg_theta", _i, [_p, _p, _p, _i, _d, _p, _p, _p]),
    ("id11b_dev_bragg_theta_adjoint", _i, [_p, _p, _p, _i, _d, _p, _p, _p]),
]


class ID11BError(RuntimeError):
    """A C-ABI call returned a non-zero status."""


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "imaged11_b200: %s is missing; build it with `python -m imaged11_b200.build`"
            % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in _SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def status_text(rc):
    return lib.id11b_status_string(rc).decode()


def check(rc, what=""):
    """Raise ID11BError for a non-zero status."""
    if rc:
        msg = "%s: %s" % (what or "imaged11_b200", status_text(rc))
        if rc == 2:
            msg += " (cudaError %d)" % lib.id11b_last_cuda_error()
        raise ID11BError(msg)


def check_last(what=""):
    """Raise for the calling thread's last layer-1 status."""
    check(lib.id11b_last_status(), what)


def exported_symbols():
    return [s[0] for s in _SIGNATURES]
