"""Host side of the FFT Poisson solver without a GPU: the library exports
every function include/bfft.h declares, descriptors the reference rejects
are rejected before any device work, and a missing device fails loudly."""
import ctypes
import os
import re

import numpy as np
import pytest

from briscola_b200 import fft
from briscola_b200.build import build_fft
from briscola_b200.mesh import DIRICHLET, EMPTY, NEUMANN, PERIODIC, Brick, geometric_points, uniform_points

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_function():
    lib = ctypes.CDLL(build_fft())
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "bfft.h")).read(), flags=re.S)
    fns = sorted(set(re.findall(r"\b(bfft_[a-z_0-9]+)\s*\(", txt)))
    assert len(fns) == 9
    assert [f for f in fns if not hasattr(lib, f)] == []
    assert set(fns) == set(fft.EXPORTED)


def _create(brick):
    L = fft.load(build_fft())
    pts = [np.ascontiguousarray(p) for p in brick.points]
    d = fft.Desc()
    for a in range(3):
        d.n[a] = len(pts[a]) - 1
        d.points[a] = pts[a].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for f in range(6):
        d.bc[f] = fft.BC[brick.bc[f]]
    h = ctypes.c_void_p()
    rc = L.bfft_create(ctypes.byref(h), ctypes.byref(d))
    if rc == 0:
        L.bfft_destroy(h)
    return rc


def test_descriptor_checks_come_before_the_device():
    u = uniform_points(16)
    # two non-uniform directions (FFTPoissonSolver.C:23-45)
    assert _create(Brick([u, geometric_points(16, 2.0), geometric_points(16, 2.0)])) == 3
    # a periodic face paired with a wall (FourierTransforms.C:219-224)
    assert _create(Brick([u, u, u], (PERIODIC, NEUMANN, NEUMANN, NEUMANN, NEUMANN, NEUMANN))) == 3
    # an empty axis with more than one cell
    assert _create(Brick([u, u, u], (NEUMANN, NEUMANN, EMPTY, EMPTY, NEUMANN, NEUMANN))) == 3
    # a transformed extent that is not a power of two: unsupported by this build
    assert _create(Brick([u, uniform_points(12), u], (DIRICHLET,) * 6)) == 7


def test_create_without_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    u = uniform_points(16)
    assert _create(Brick([u, u, u], (DIRICHLET,) * 6)) == 6
    with pytest.raises(fft.FatalError):
        fft.FFTPoissonSolver(Brick([u, u, u], (DIRICHLET,) * 6))


def test_runtime_table():
    with pytest.raises(fft.FatalError, match="Valid Poisson solvers"):
        fft.New({"type": "nope"}, None)
    assert fft.POISSON_SOLVERS["FFT"] is fft.FFTPoissonSolver
