"""The FFT Poisson solver on B200 (``include/bfft.h``, ``csrc/bfft.cu``).

Mirrors the reference's ``FFTPoissonSolver`` (PoissonSolver type ``"FFT"``,
src/briscolaFiniteVolume/solvers/PoissonSolvers/FFTPoissonSolver/
FFTPoissonSolver.H:44-121): a direct solve of the constant-coefficient
Poisson equation on one rectilinear brick with at least two uniform
directions, by trigonometric / real Fourier transforms along the uniform
directions and a tridiagonal solve per mode along the third.

``solve(x, b)`` leaves in ``x`` the solution of Laplacian(x) = -b with the
brick's face values (Dirichlet values, Neumann gradients); with ``ddt`` it
solves Laplacian(x) - x/dt' = -b - x_old/dt', dt' = dt * dtFrac, as the
reference does (FFTPoissonSolver.C:88-131).  A ``lambda`` coefficient is
refused, as in the reference (FFTPoissonSolver.C:97-104).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .mesh import DIRICHLET, EMPTY, NEUMANN, PERIODIC, Brick, Mesh
from .solvers import FatalError

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libbfft.so")
EXPORTED = ("bfft_create", "bfft_destroy", "bfft_set_stream", "bfft_solve", "bfft_solve_direction",
            "bfft_last_error", "bfft_split_lambda0", "bfft_split_source", "bfft_axpby")
BC = {DIRICHLET: 0, NEUMANN: 1, PERIODIC: 2, EMPTY: 3}
DEVICE_PTRS = 1


class Desc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int * 3),
        ("points", ctypes.POINTER(ctypes.c_double) * 3),
        ("bc", ctypes.c_int * 6),
        ("value", ctypes.c_double * 6),
        ("device", ctypes.c_int),
    ]


_lib = None


def load(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"FFT solver library not found at {path}; build it with "
                           "`python -c 'import __graft_entry__ as g; g.build()'` (there is no CPU fallback)")
    L = ctypes.CDLL(path)
    missing = [s for s in EXPORTED if not hasattr(L, s)]
    if missing:
        raise RuntimeError(f"{path} lacks exported symbols: {missing}")
    vp = ctypes.c_void_p
    L.bfft_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Desc)]
    L.bfft_destroy.argtypes = [vp]
    L.bfft_destroy.restype = None
    L.bfft_set_stream.argtypes = [vp, vp]
    L.bfft_solve.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_int]
    L.bfft_solve_direction.argtypes = [vp]
    L.bfft_last_error.argtypes = [vp]
    L.bfft_last_error.restype = ctypes.c_char_p
    L.bfft_split_lambda0.argtypes = [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_double)]
    L.bfft_split_source.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_double, vp]
    L.bfft_axpby.argtypes = [vp, ctypes.c_double, vp, ctypes.c_double, vp, vp]
    _lib = L
    return L


def _brick(mesh) -> Brick:
    if isinstance(mesh, Mesh):
        if len(mesh.bricks) != 1:
            raise FatalError("the FFT solver takes a single-brick mesh")
        return mesh.bricks[0]
    return mesh


class FFTPoissonSolver:
    """The "FFT" Poisson solver of one brick.  ``values``: the Dirichlet
    value or Neumann gradient of each face (x-lo, x-hi, y-lo, ...); by
    default the brick's face values."""

    typeName = "FFT"

    def __init__(self, mesh, values=None, device: int = 0):
        self.brick = _brick(mesh)
        self.N = self.brick.N
        self.values = tuple(float(v) for v in (self.brick.values if values is None else values))
        for f in self.brick.bc:
            if f not in BC:
                raise FatalError(f"Incompatible boundary condition {f}")
        self._lib = load()
        self._pts = [np.ascontiguousarray(p, dtype=np.float64) for p in self.brick.points]
        d = Desc()
        for a in range(3):
            d.n[a] = self.N[a]
            d.points[a] = self._pts[a].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        for f in range(6):
            d.bc[f] = BC[self.brick.bc[f]]
            d.value[f] = self.values[f]
        d.device = int(device)
        self.device = int(device)
        self.h = ctypes.c_void_p()
        rc = self._lib.bfft_create(ctypes.byref(self.h), ctypes.byref(d))
        if rc != 0:
            raise FatalError(f"bfft_create failed with status {rc}")
        self._stream = None

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.bfft_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def solve_direction(self) -> int:
        return self._lib.bfft_solve_direction(self.h)

    def _check(self, rc, what):
        if rc != 0:
            raise FatalError(f"{what}: status {rc} {self._lib.bfft_last_error(self.h).decode()}".strip())

    def set_stream(self, stream: int):
        self._check(self._lib.bfft_set_stream(self.h, ctypes.c_void_p(stream)), "bfft_set_stream")
        self._stream = stream

    def solve(self, x, b, lam=None, ddt: bool = False, dt: float = 0.0, dtFrac: float = 1.0, x_old=None):
        """x (n0, n1, n2) <- the solution for right-hand side b.  Host numpy
        arrays, or CUDA tensors (solved on torch's current stream)."""
        if lam is not None:
            raise FatalError("FFT Poisson solver does not support use of lambda argument in solve function.")
        shift = 0.0
        if ddt:
            if dt <= 0.0 or x_old is None:
                raise FatalError("a ddt solve needs dt > 0 and the old-time field")
            shift = 1.0 / (dt * dtFrac)
        n = int(np.prod(self.N))
        try:
            import torch
            on_device = isinstance(x, torch.Tensor) and x.is_cuda
        except ImportError:
            torch = None
            on_device = False
        if on_device:
            for t in (x, b) + ((x_old,) if x_old is not None else ()):
                if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == n):
                    raise FatalError("device arrays must be contiguous float64 CUDA tensors of the mesh size")
            s = torch.cuda.current_stream().cuda_stream
            if s != self._stream:
                self.set_stream(s)
            xo = x_old.data_ptr() if x_old is not None else None
            self._check(self._lib.bfft_solve(self.h, b.data_ptr(), x.data_ptr(), xo, shift, DEVICE_PTRS),
                        "bfft_solve")
            return x
        bh = np.ascontiguousarray(b, dtype=np.float64)
        if bh.size != n:
            raise FatalError("b does not match the mesh")
        xh = x if (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous) else None
        out = xh if xh is not None else np.empty(self.N)
        xo = None
        if x_old is not None:
            xo_arr = np.ascontiguousarray(x_old, dtype=np.float64)
            xo = xo_arr.ctypes.data
        self._check(self._lib.bfft_solve(self.h, bh.ctypes.data, out.ctypes.data, xo, shift, 0), "bfft_solve")
        if xh is None and x is not None:
            x[...] = out.reshape(np.shape(x))
        return out


# the reference's PoissonSolver runtime table, for the types this package
# implements (PoissonSolver.H run-time selection by "type")
POISSON_SOLVERS = {FFTPoissonSolver.typeName: FFTPoissonSolver}


def New(d: dict, mesh, **kw):
    t = str(d.get("type", ""))
    if t not in POISSON_SOLVERS:
        raise FatalError(f"Unknown Poisson solver {t}\n\nValid Poisson solvers are:\n{sorted(POISSON_SOLVERS)}")
    return POISSON_SOLVERS[t](mesh, **kw)
