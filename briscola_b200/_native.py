"""ctypes bindings of ``libbmg.so`` (the C ABI in ``include/bmg.h``).

The shared library is built in-tree (``briscola_b200/_lib/libbmg.so``) by
``briscola_b200.build.build_native``.  There is no fallback: if the library
is missing or no sm_100 device is present the calls fail with an error.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbmg.so")

# status codes (bmg_status)
OK, NOT_CONVERGED, NAN_DETECTED, BAD_ARG, CUDA_ERROR, TIMEOUT, NO_DEVICE, UNSUPPORTED = range(8)
BC_NEUMANN, BC_PERIODIC, BC_DIRICHLET = 0, 1, 2
CYCLE = {"V": 0, "W": 1, "F": 2}
SMOOTHER = {"rbgs": 0, "jac": 1, "jacobi": 1}
PRECISION = {"fp64": 0, "mixed": 1}
KRYLOV = {"none": 0, "fcg": 1}
CRITERION = {"initial": 0, "rhs": 1}
COARSE_MODE = {"direct": 0, "smooth": 1}
RESTRICT = {"linear": 0, "average": 1}
PROLONG = {"linear": 0, "injection": 1}
ROW_LAYOUT = {"split": 0, "natural": 1}
LEVEL_MODE = {"replace": 0, "guess": 1}
DEVICE_PTRS, ZERO_GUESS, PER_VOLUME = 1, 2, 4

# Every function the header declares; the loader checks they are exported.
EXPORTED = (
    "bmg_default_options", "bmg_create", "bmg_destroy", "bmg_set_coefficients", "bmg_set_stream",
    "bmg_set_options", "bmg_solve", "bmg_num_cells", "bmg_num_levels", "bmg_level_shape",
    "bmg_status_string", "bmg_last_error", "bmg_level_upload", "bmg_level_download",
    "bmg_op_colour_pass", "bmg_op_smooth", "bmg_op_residual", "bmg_op_residual_restrict",
    "bmg_op_prolong_correct", "bmg_op_coarse_solve", "bmg_coarse_level_index",
    "bmg_residual_norm_noalloc", "bmg_level_tuning", "bmg_set_level_tuning", "bmg_project_rhs",
    "bmg_project_correct", "bmg_set_level_solver",
)

# int (*bmg_level_solver)(void* user, void* stream, const float* rhs, float* x, const int n[3])
LEVEL_SOLVER = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.POINTER(ctypes.c_int))


class Brick(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int * 3),
        ("points", ctypes.POINTER(ctypes.c_double) * 3),
        ("bc", ctypes.c_int * 6),
        ("origin", ctypes.c_int * 3),
        ("value", ctypes.c_double * 6),
        ("transform", ctypes.c_int * 3),
    ]


class MeshDesc(ctypes.Structure):
    _fields_ = [("n_bricks", ctypes.c_int), ("bricks", ctypes.POINTER(Brick))]


class Options(ctypes.Structure):
    _fields_ = [
        ("rel_tol", ctypes.c_double),
        ("abs_tol", ctypes.c_double),
        ("min_iter", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("n_pre", ctypes.c_int),
        ("n_post", ctypes.c_int),
        ("cycle_type", ctypes.c_int),
        ("coarse_level", ctypes.c_int),
        ("smoother", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("use_graph", ctypes.c_int),
        ("remove_mean", ctypes.c_int),
        ("fused", ctypes.c_int),
        ("autotune", ctypes.c_int),
        ("device", ctypes.c_int),
        ("timeout_ms", ctypes.c_double),
        ("krylov", ctypes.c_int),
        ("criterion", ctypes.c_int),
        ("fused_chunk", ctypes.c_int),
        ("fuse_coarse", ctypes.c_int),
        ("coarse_mode", ctypes.c_int),
        ("restrict_scheme", ctypes.c_int),
        ("prolong_scheme", ctypes.c_int),
        ("row_layout", ctypes.c_int),
        ("fuse_first", ctypes.c_int),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("cycles", ctypes.c_int),
        ("outer_iterations", ctypes.c_int),
        ("initial_residual", ctypes.c_double),
        ("final_residual", ctypes.c_double),
        ("rel_residual", ctypes.c_double),
        ("final_l2", ctypes.c_double),
        ("norm_factor", ctypes.c_double),
        ("ms", ctypes.c_float),
        ("kernel_launches", ctypes.c_long),
        ("rhs_rel_residual", ctypes.c_double),
    ]


_lib = None


def load(path: str = LIB_PATH):
    """Load the native library (once) and declare argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"native solver library not found at {path}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (there is no CPU fallback)"
        )
    L = ctypes.CDLL(path)
    missing = [s for s in EXPORTED if not hasattr(L, s)]
    if missing:
        raise RuntimeError(f"{path} lacks exported symbols: {missing}")
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.bmg_default_options.argtypes = [ctypes.POINTER(Options)]
    L.bmg_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(MeshDesc), ctypes.POINTER(Options)]
    L.bmg_destroy.argtypes = [vp]
    L.bmg_destroy.restype = None
    L.bmg_set_coefficients.argtypes = [vp, dp, dp, dp]
    L.bmg_set_stream.argtypes = [vp, vp]
    L.bmg_set_options.argtypes = [vp, ctypes.POINTER(Options)]
    L.bmg_solve.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(Report)]
    L.bmg_num_cells.argtypes = [vp]
    L.bmg_num_cells.restype = ctypes.c_long
    L.bmg_num_levels.argtypes = [vp]
    L.bmg_level_shape.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip]
    L.bmg_status_string.argtypes = [ctypes.c_int]
    L.bmg_status_string.restype = ctypes.c_char_p
    L.bmg_last_error.argtypes = [vp]
    L.bmg_last_error.restype = ctypes.c_char_p
    L.bmg_level_upload.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    L.bmg_level_download.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    L.bmg_op_colour_pass.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.bmg_op_smooth.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.bmg_op_residual.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
    L.bmg_op_residual_restrict.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.bmg_op_prolong_correct.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.bmg_op_coarse_solve.argtypes = [vp, ctypes.c_int]
    L.bmg_coarse_level_index.argtypes = [vp]
    L.bmg_residual_norm_noalloc.argtypes = [vp, vp, ip, vp, vp, vp, ip, vp, vp]
    L.bmg_level_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip]
    L.bmg_set_level_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.bmg_project_rhs.argtypes = [vp, vp, vp, vp, ctypes.c_double, vp, ctypes.c_int]
    L.bmg_project_correct.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_double]
    L.bmg_set_level_solver.argtypes = [vp, ctypes.c_int, LEVEL_SOLVER, vp, ctypes.c_int]
    _lib = L
    return L


def status_string(code: int) -> str:
    return load().bmg_status_string(int(code)).decode()
