"""The split Poisson solver on B200.

Mirrors the reference's ``splitPoissonSolver`` (PoissonSolver type
``"split"``, src/briscolaFiniteVolume/solvers/PoissonSolvers/
splitPoissonSolver/splitPoissonSolver.C:15-155): the variable-coefficient
equation -div(lambda grad x) = b is solved by a prediction from two old time
levels, an optional preconditioner solve of the full variable-coefficient
problem, and nCorr corrections that each solve the constant-coefficient
equation -laplacian(x) = b / lambda0 + div((lambda / lambda0 - 1) grad x)
with lambda0 = max lambda (the pressure splitting of Dodd and Ferrante).

Here the corrections run on the GPU FFT solver (``include/bfft.h``:
``bfft_split_lambda0``, ``bfft_split_source``, ``bfft_solve``) and the
preconditioner, when the dictionary names one, is the GPU multigrid with the
face coefficients (``include/bmg.h``).  Fields are torch CUDA tensors, or
host arrays that are copied to the device.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import fft
from .mesh import Mesh
from .solvers import Context, FatalError, _switch, make_options


class SplitPoissonSolver:
    """``d``: the solver dictionary (``solver`` sub-dictionary of type FFT,
    optional ``preconditioner`` sub-dictionary of a GPUMG solver, ``nCorr``,
    ``prediction``); ``values``: the face values of the boundary conditions
    (Dirichlet values, Neumann gradients; by default the brick's)."""

    typeName = "split"

    def __init__(self, mesh, d: dict, values=None, device: int = 0):
        d = dict(d)
        sd = d.get("solver")
        if sd is None:
            raise FatalError("the split Poisson solver needs a solver sub-dictionary")
        if str(sd.get("type", "")) != fft.FFTPoissonSolver.typeName:
            raise FatalError(f"the split solver's inner solver must be of type FFT, not {sd.get('type')}")
        self.mesh = mesh if isinstance(mesh, Mesh) else Mesh([mesh])
        self.brick = self.mesh.bricks[0]
        if values is not None:
            # the face values of both the FFT corrections and the multigrid
            # preconditioner
            self.brick = dataclasses.replace(self.brick, values=tuple(float(v) for v in values))
            self.mesh = Mesh([self.brick])
        self.inner = fft.FFTPoissonSolver(self.brick, None, device)
        self.device = int(device)
        # splitPoissonSolver.C:31-52
        self.nCorr = int(d.get("nCorr", 1))
        if self.nCorr < 1:
            raise FatalError("nCorr must be at least 1")
        self.prediction = _switch(d.get("prediction", True))
        self.pre = None
        pd = d.get("preconditioner")
        if pd is not None:
            if str(pd.get("type", "")) not in ("GPUMG", "MG"):
                raise FatalError(f"the split solver's preconditioner must be GPUMG, not {pd.get('type')}")
            opts = {k: v for k, v in dict(pd).items() if k != "type"}
            self.pre = Context(self.mesh, make_options(dict(opts, device=self.device)))
        self._lib = fft.load()
        self._V = None
        self._pre_set = False

    def close(self):
        self.inner.close()
        if self.pre is not None:
            self.pre.close()

    def _check(self, rc, what):
        self.inner._check(rc, what)

    def solve(self, x, b, lam, ddt: bool = False, dt: float = 0.0, dtFrac: float = 1.0, dt0: float = 0.0,
              x_old=None, x_oldold=None, constMatrix: bool = False):
        """x <- the split solution; lam: the three face-coefficient arrays
        ((n0+1, n1, n2), (n0, n1+1, n2), (n0, n1, n2+1)).  constMatrix: the
        coefficients are those of the previous solve, so the preconditioner
        keeps its operator (the reference's solve(sys, constMatrix))."""
        import torch

        if lam is None:
            raise FatalError("Poisson equation has no coefficient so it cannot be split.")
        dev = torch.device("cuda", self.device)
        on_device = isinstance(x, torch.Tensor) and x.is_cuda

        def to_dev(a):
            if a is None:
                return None
            t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
            return t.to(dev, dtype=torch.float64).contiguous()

        xd = x if on_device else to_dev(x)
        bd = to_dev(b)
        lams = [to_dev(l) for l in lam]
        stream = torch.cuda.current_stream(dev).cuda_stream
        if self.inner._stream != stream:
            self.inner.set_stream(stream)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

        # prediction from two old levels (splitPoissonSolver.C:75-84)
        if self.prediction:
            if x_old is None or x_oldold is None or dt0 <= 0.0:
                raise FatalError("the prediction needs the two old time levels and the old time step")
            r = dt * dtFrac / dt0
            xo, xoo = to_dev(x_old), to_dev(x_oldold)
            self._check(self._lib.bfft_axpby(self.inner.h, 1.0 + r, ptr(xo), -r, ptr(xoo), ptr(xd)), "bfft_axpby")

        # preconditioner: the variable-coefficient problem on the GPU
        # multigrid, A x = -V b (linearSystem.C:547-556), from the current x
        if self.pre is not None:
            if ddt:
                raise FatalError("the multigrid preconditioner takes no ddt term")
            if self._V is None:
                self._V = torch.from_numpy(self.brick.cell_volumes()).to(dev)
            self.pre.set_stream(stream)
            if not (constMatrix and self._pre_set):
                self.pre.set_coefficients([l.cpu().numpy() for l in lams])
                self._pre_set = True
            bsys = -(self._V * bd.view(self.brick.N)).reshape(-1).contiguous()
            self.pre.solve(bsys, xd.view(-1), zero_guess=False)

        lambda0 = ctypes.c_double()
        self._check(self._lib.bfft_split_lambda0(self.inner.h, ptr(lams[0]), ptr(lams[1]), ptr(lams[2]),
                                                 ctypes.byref(lambda0)), "bfft_split_lambda0")
        bhat = torch.empty_like(bd)
        for _ in range(self.nCorr):
            self._check(self._lib.bfft_split_source(self.inner.h, ptr(xd), ptr(bd), ptr(lams[0]), ptr(lams[1]),
                                                    ptr(lams[2]), lambda0.value, ptr(bhat)), "bfft_split_source")
            self.inner.solve(xd, bhat, ddt=ddt, dt=dt, dtFrac=dtFrac, x_old=to_dev(x_old) if ddt else None)
        if not on_device:
            out = xd.cpu().numpy().reshape(np.shape(x))
            x[...] = out
        self.lambda0 = lambda0.value
        return x


def New(d: dict, mesh, **kw):
    """PoissonSolver run-time selection for the types this package has."""
    t = str(d.get("type", ""))
    if t == SplitPoissonSolver.typeName:
        return SplitPoissonSolver(mesh, d, **kw)
    return fft.New(d, mesh, **kw)
