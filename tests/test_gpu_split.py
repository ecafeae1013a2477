"""The split Poisson solver on the GPU (briscola_b200/split.py over the FFT
solver's split kernels) against the CPU restatement of
splitPoissonSolver.C (oracle/fft_oracle.py): the modified source and the
largest coefficient on mixed faces, whole corrections without a
preconditioner, the prediction from two old levels, and the GPU multigrid as
preconditioner on a density-ratio-10 coefficient."""
import numpy as np
import pytest

from briscola_b200 import split
from briscola_b200.mesh import DIRICHLET, NEUMANN, PERIODIC, Brick, geometric_points, uniform_points
from oracle import fft_oracle as F

pytestmark = pytest.mark.gpu

D, N, P = DIRICHLET, NEUMANN, PERIODIC


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def lambdas(n, ratio, rng, periodic):
    lam = []
    for d in range(3):
        shape = list(n)
        shape[d] += 1
        a = 1.0 + (ratio - 1.0) * rng.random(shape)
        if periodic[d]:
            idx = [slice(None)] * 3
            first = [slice(None)] * 3
            idx[d], first[d] = -1, 0
            a[tuple(idx)] = a[tuple(first)]
        lam.append(a)
    return lam


def test_modified_source_and_lambda0_on_mixed_faces():
    torch = pytest.importorskip("torch")
    n = (16, 24, 8)
    pts = [uniform_points(16), geometric_points(24, 2.0), uniform_points(8)]
    bc = (D, N, N, D, P, P)
    vals = (0.5, -1.0, 2.0, 0.25, 0.0, 0.0)
    rng = np.random.default_rng(2)
    lam = lambdas(n, 3.0, rng, (False, False, True))
    x = rng.standard_normal(n)
    b = rng.standard_normal(n)
    s = split.SplitPoissonSolver(Brick(pts, bc), {"solver": {"type": "FFT"}, "prediction": "off"}, vals)
    lib, h = s._lib, s.inner.h
    import ctypes

    dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    xd, bd, ld = dv(x), dv(b), [dv(l) for l in lam]
    out = torch.empty_like(bd)
    l0 = ctypes.c_double()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert lib.bfft_split_lambda0(h, p(ld[0]), p(ld[1]), p(ld[2]), ctypes.byref(l0)) == 0
    assert l0.value == max(l.max() for l in lam)
    assert lib.bfft_split_source(h, p(xd), p(bd), p(ld[0]), p(ld[1]), p(ld[2]), l0.value, p(out)) == 0
    torch.cuda.synchronize()
    ref = F.split_source(x, b, lam, l0.value, pts, bc, vals)
    assert rel(out.cpu().numpy(), ref) <= 1e-13
    s.close()


def test_corrections_match_the_oracle():
    n = (16, 32, 16)
    pts = [uniform_points(16), geometric_points(32, 2.0), uniform_points(16)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(3)
    lam = lambdas(n, 2.0, rng, (True, False, True))
    b = rng.standard_normal(n)
    V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
    b -= (b * V).sum() / V.sum()
    x0 = rng.standard_normal(n)
    s = split.New({"type": "split", "solver": {"type": "FFT"}, "nCorr": 4, "prediction": "off"}, Brick(pts, bc))
    x = x0.copy()
    s.solve(x, b, lam)
    ref = F.split_solve(x0, b, lam, pts, bc, n_corr=4)
    assert rel(x, ref) <= 1e-11
    s.close()


def test_prediction_from_two_old_levels():
    torch = pytest.importorskip("torch")
    n = (8, 16, 8)
    pts = [uniform_points(8), geometric_points(16, 2.0), uniform_points(8)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(4)
    lam = lambdas(n, 1.5, rng, (True, False, True))
    b = rng.standard_normal(n)
    b -= b.mean()
    xo, xoo = rng.standard_normal(n), rng.standard_normal(n)
    s = split.SplitPoissonSolver(Brick(pts, bc), {"solver": {"type": "FFT"}, "nCorr": 1})
    x = np.zeros(n)
    dt, dt0 = 0.02, 0.01
    s.solve(x, b, lam, dt=dt, dt0=dt0, x_old=xo, x_oldold=xoo)
    guess = (1.0 + dt / dt0) * xo - dt / dt0 * xoo
    assert rel(x, F.split_solve(guess, b, lam, pts, bc, n_corr=1)) <= 1e-11
    with pytest.raises(split.FatalError):
        s.solve(x, b, None)  # no coefficient: the reference refuses to split
    s.close()


def test_multigrid_preconditioner_reduces_the_residual():
    n = (32, 32, 32)
    pts = [uniform_points(32), geometric_points(32, 3.0), uniform_points(32)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(5)
    lam = lambdas(n, 10.0, rng, (True, False, True))
    b = rng.standard_normal(n)
    V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
    b -= (b * V).sum() / V.sum()
    res = {}
    for name, extra in (("plain", {}),
                        ("mg", {"preconditioner": {"type": "GPUMG", "maxIter": 3, "relTol": 0, "tolerance": 0,
                                                   "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2,
                                                   "coarseLevel": 1}})):
        s = split.SplitPoissonSolver(Brick(pts, bc), dict({"solver": {"type": "FFT"}, "nCorr": 2,
                                                           "prediction": "off"}, **extra))
        x = np.zeros(n)
        s.solve(x, b, lam)
        r = F.variable_residual(x, b, lam, pts, bc)
        res[name] = np.abs(r - (r * V).sum() / V.sum()).max()
        s.close()
    assert res["mg"] < 0.2 * res["plain"], res
