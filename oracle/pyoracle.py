"""ctypes view of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``bmg_oracle.cpp``) restates the reference multigrid solve on the
CPU; see the header of ``bmg_oracle.h`` for the reference files it follows.
Only the tests, the smoke check and the CPU-baseline leg of ``bench.py`` use
this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libbmg_oracle.so")


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
        ("coarse_direct", ctypes.c_int),
        ("smoother", ctypes.c_int),
        ("stale_residual", ctypes.c_int),
        ("restrict_average", ctypes.c_int),
        ("prolong_injection", ctypes.c_int),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("initial_residual", ctypes.c_double),
        ("final_residual", ctypes.c_double),
        ("norm_factor", ctypes.c_double),
        ("final_l2", ctypes.c_double),
        ("b_l2", ctypes.c_double),
    ]


_CYCLES = {"V": 0, "W": 1, "F": 2}
_SMOOTHERS = {"rbgs": 0, "jac": 1, "jacobi": 1}
_lib = None


def build() -> str:
    """Compile the oracle library (make) if it is missing; return its path."""
    if not os.path.exists(_SO):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.bmgo_create.restype = vp
        L.bmgo_create.argtypes = [ip, dp, dp, dp, ip, ctypes.c_int]
        L.bmgo_destroy.argtypes = [vp]
        L.bmgo_set_faces.argtypes = [vp, ip, dp]
        L.bmgo_num_levels.argtypes = [vp]
        L.bmgo_level_shape.argtypes = [vp, ctypes.c_int, ip]
        L.bmgo_level_ratio.argtypes = [vp, ctypes.c_int, ip]
        L.bmgo_cell_centres.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.bmgo_cell_volumes.argtypes = [vp, ctypes.c_int, dp]
        L.bmgo_set_lambda.argtypes = [vp, dp, dp, dp]
        L.bmgo_get_lambda.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.bmgo_default_options.argtypes = [ctypes.POINTER(Options)]
        L.bmgo_assemble.argtypes = [vp, ctypes.POINTER(Options)]
        L.bmgo_get_matrix.argtypes = [vp, ctypes.c_int, dp]
        L.bmgo_solve.argtypes = [vp, ctypes.POINTER(Options), dp, dp, ctypes.POINTER(Report), dp, ctypes.c_int]
        L.bmgo_residual.argtypes = [vp, ctypes.c_int, dp, dp, dp]
        L.bmgo_smooth.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        L.bmgo_colour_pass.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.bmgo_restrict.argtypes = [vp, ctypes.c_int, dp, dp, ctypes.c_int]
        L.bmgo_prolong.argtypes = [vp, ctypes.c_int, dp, dp, ctypes.c_int]
        L.bmgo_prolong_ghosted.argtypes = [vp, ctypes.c_int, dp, dp, ctypes.c_int]
        L.bmgo_coarse_solve.argtypes = [vp, ctypes.c_int, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def options(**kw) -> Options:
    o = Options()
    lib().bmgo_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if k == "cycle_type" and isinstance(v, str):
            v = _CYCLES[v]
        if k == "smoother" and isinstance(v, str):
            v = _SMOOTHERS[v]
        setattr(o, k, v)
    return o


class Oracle:
    """One rectilinear brick: ``points`` is a list of three vertex-coordinate
    arrays (N_d + 1 each); ``periodic`` flags per axis (walls otherwise)."""

    def __init__(self, points, periodic=(False, False, False), nthreads: int = 0, dirichlet=None,
                 values=None):
        self.points = [np.ascontiguousarray(p, dtype=np.float64) for p in points]
        self.N = tuple(len(p) - 1 for p in self.points)
        N = (ctypes.c_int * 3)(*self.N)
        per = (ctypes.c_int * 3)(*[int(bool(x)) for x in periodic])
        self.periodic = tuple(bool(x) for x in periodic)
        self._p = lib().bmgo_create(N, *[_dp(p) for p in self.points], per, int(nthreads))
        if dirichlet is not None:
            self.set_faces(dirichlet, values)

    def set_faces(self, dirichlet, values=None):
        """Dirichlet walls (flags per face x-lo, x-hi, y-lo, ...) with uniform
        values; the other walls stay Neumann."""
        self._dval = np.ascontiguousarray(values if values is not None else np.zeros(6), dtype=np.float64)
        flags = (ctypes.c_int * 6)(*[int(bool(x)) for x in dirichlet])
        if lib().bmgo_set_faces(self._p, flags, _dp(self._dval)) != 0:
            raise ValueError("a Dirichlet face on a periodic axis")

    def __del__(self):
        if getattr(self, "_p", None):
            lib().bmgo_destroy(self._p)
            self._p = None

    # --- hierarchy -------------------------------------------------------
    @property
    def num_levels(self) -> int:
        return lib().bmgo_num_levels(self._p)

    def shape(self, l: int):
        n = (ctypes.c_int * 3)()
        lib().bmgo_level_shape(self._p, l, n)
        return tuple(n)

    def ratio(self, l: int):
        n = (ctypes.c_int * 3)()
        lib().bmgo_level_ratio(self._p, l, n)
        return tuple(n)

    def centres(self, l: int, axis: int) -> np.ndarray:
        out = np.zeros(self.shape(l)[axis] + 2)
        lib().bmgo_cell_centres(self._p, l, axis, _dp(out))
        return out

    def volumes(self, l: int) -> np.ndarray:
        out = np.zeros(self.shape(l))
        lib().bmgo_cell_volumes(self._p, l, _dp(out))
        return out

    # --- operator --------------------------------------------------------
    def set_lambda(self, lx=None, ly=None, lz=None):
        if lx is None:
            lib().bmgo_set_lambda(self._p, None, None, None)
            return
        self._lam = [np.ascontiguousarray(a, dtype=np.float64) for a in (lx, ly, lz)]
        lib().bmgo_set_lambda(self._p, *[_dp(a) for a in self._lam])

    def get_lambda(self, l: int, fd: int) -> np.ndarray:
        n = list(self.shape(l))
        n[fd] += 1
        out = np.zeros(n)
        lib().bmgo_get_lambda(self._p, l, fd, _dp(out))
        return out

    def assemble(self, **kw):
        o = options(**kw)
        lib().bmgo_assemble(self._p, ctypes.byref(o))

    def matrix(self, l: int) -> np.ndarray:
        out = np.zeros(self.shape(l) + (7,))
        lib().bmgo_get_matrix(self._p, l, _dp(out))
        return out

    # --- solve -----------------------------------------------------------
    def solve(self, b: np.ndarray, x0: np.ndarray | None = None, max_hist: int = 1000, **kw):
        o = options(**kw)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        rep = Report()
        hist = np.zeros(max_hist)
        rc = lib().bmgo_solve(self._p, ctypes.byref(o), _dp(b), _dp(x), ctypes.byref(rep), _dp(hist), max_hist)
        return x, rep, hist[: min(rep.iterations, max_hist)], rc

    # --- building blocks -------------------------------------------------
    def residual(self, l, x, b):
        r = np.zeros(self.shape(l))
        lib().bmgo_residual(self._p, l, _dp(np.ascontiguousarray(x, dtype=np.float64)),
                            _dp(np.ascontiguousarray(b, dtype=np.float64)), _dp(r))
        return r

    def smooth(self, l, x, b, sweeps=1, smoother="rbgs"):
        x = np.array(x, dtype=np.float64, copy=True)
        lib().bmgo_smooth(self._p, l, _SMOOTHERS[smoother], sweeps, _dp(x),
                          _dp(np.ascontiguousarray(b, dtype=np.float64)))
        return x

    def colour_pass(self, l, colour, x, b):
        x = np.array(x, dtype=np.float64, copy=True)
        lib().bmgo_colour_pass(self._p, l, colour, _dp(x), _dp(np.ascontiguousarray(b, dtype=np.float64)))
        return x

    def restrict(self, lf, fine, scale=True):
        out = np.zeros(self.shape(lf + 1))
        lib().bmgo_restrict(self._p, lf, _dp(np.ascontiguousarray(fine, dtype=np.float64)), _dp(out), int(scale))
        return out

    def prolong(self, lf, coarse, fine=None, op="+="):
        fine = np.zeros(self.shape(lf)) if fine is None else np.array(fine, dtype=np.float64, copy=True)
        lib().bmgo_prolong(self._p, lf, _dp(np.ascontiguousarray(coarse, dtype=np.float64)), _dp(fine),
                           1 if op == "+=" else 0)
        return fine

    def prolong_ghosted(self, lf, coarse_g, fine=None, op="="):
        fine = np.zeros(self.shape(lf)) if fine is None else np.array(fine, dtype=np.float64, copy=True)
        lib().bmgo_prolong_ghosted(self._p, lf, _dp(np.ascontiguousarray(coarse_g, dtype=np.float64)),
                                   _dp(fine), 1 if op == "+=" else 0)
        return fine

    def coarse_solve(self, l, b):
        x = np.zeros(self.shape(l))
        lib().bmgo_coarse_solve(self._p, l, _dp(np.ascontiguousarray(b, dtype=np.float64)), _dp(x))
        return x
