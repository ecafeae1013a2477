"""The CPU restatement of the reference's FFT Poisson solver (oracle/
fft_oracle.py): its transforms against their FFTW definitions written as
direct sums, and the whole solve against the reference's own known-answer
test (Test-FFTPoissonSolver.C: random right-hand side, mixed Dirichlet /
Neumann faces with nonzero values, a stretched direction, pointwise residual
of the discrete Laplacian <= 1e-10)."""
import numpy as np
import pytest

from briscola_b200.mesh import geometric_points, uniform_points
from oracle import fft_oracle as F

D, N, P = F.DIRICHLET, F.NEUMANN, F.PERIODIC


def direct(kind, x):
    n = len(x)
    k = np.arange(n)[:, None]
    m = np.arange(n)[None, :]
    if kind == "REDFT10":
        return 2 * (x * np.cos(np.pi * (m + 0.5) * k / n)).sum(1)
    if kind == "REDFT01":
        return x[0] + 2 * (x[1:] * np.cos(np.pi * m[:, 1:] * (k + 0.5) / n)).sum(1)
    if kind == "RODFT10":
        return 2 * (x * np.sin(np.pi * (m + 0.5) * (k + 1) / n)).sum(1)
    if kind == "RODFT01":
        return (-1.0) ** k[:, 0] * x[-1] + 2 * (x[:-1] * np.sin(np.pi * (m[:, :-1] + 1) * (k + 0.5) / n)).sum(1)
    if kind == "REDFT11":
        return 2 * (x * np.cos(np.pi * (m + 0.5) * (k + 0.5) / n)).sum(1)
    if kind == "RODFT11":
        return 2 * (x * np.sin(np.pi * (m + 0.5) * (k + 0.5) / n)).sum(1)
    if kind == "R2HC":
        y = (x * np.exp(-2j * np.pi * m * k / n)).sum(1)
        out = np.empty(n)
        out[:n // 2 + 1] = y.real[:n // 2 + 1]
        for q in range(1, (n + 1) // 2):
            out[n - q] = y.imag[q]
        return out
    raise KeyError(kind)


@pytest.mark.parametrize("n", [1, 2, 7, 8, 16])
def test_transforms_match_fftw_definitions(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    pairs = {F.PAIR_DD: ("RODFT10", "RODFT01"), F.PAIR_NN: ("REDFT10", "REDFT01"),
             F.PAIR_DN: ("RODFT11", "RODFT11"), F.PAIR_ND: ("REDFT11", "REDFT11")}
    for code, (fw, bw) in pairs.items():
        assert np.allclose(F.forward(x, 0, code), direct(fw, x), atol=1e-12)
        assert np.allclose(F.backward(x, 0, code), direct(bw, x), atol=1e-12)
        # backward(forward(x)) = 2N x
        assert np.allclose(F.backward(F.forward(x, 0, code), 0, code), 2 * n * x, atol=1e-11)
    assert np.allclose(F.forward(x, 0, F.PAIR_CC), direct("R2HC", x), atol=1e-12)
    assert np.allclose(F.backward(F.forward(x, 0, F.PAIR_CC), 0, F.PAIR_CC), n * x, atol=1e-11)


# applications/test/FFTPoissonSolver: 16 x 64 x 32 cells on the unit cube,
# geometric grading (1 1 1), (2 1 1), (1 2 1), (1 1 2); faces x: Dirichlet 1
# and 2, y: Neumann 3 and 4, z: Neumann 5 and Dirichlet 6
REF_BC = (D, D, N, N, N, D)
REF_VALUES = (1.0, 2.0, 3.0, 4.0, 5.0, 6.0)


def ref_case(stretch, seed=123):
    n = (16, 64, 32)
    pts = [geometric_points(n[d], stretch[d]) for d in range(3)]
    rng = np.random.default_rng(seed)
    f = 100.0 * rng.random(n) - 0.5
    f -= f.mean()
    return pts, f


@pytest.mark.parametrize("stretch", [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2)])
def test_known_answer_mixed_faces(stretch):
    pts, f = ref_case(stretch)
    x = F.solve(f, pts, REF_BC, REF_VALUES)
    r = F.laplacian_residual(x, f, pts, REF_BC, REF_VALUES)
    assert np.abs(r).max() <= 1e-10 * max(1.0, np.abs(f).max() / 100.0)
    assert F.solve_direction(pts, f.shape) == (list(stretch).index(2) if 2 in stretch else 0)


@pytest.mark.parametrize("bc", [
    (P, P, N, N, P, P),   # the channel: periodic x, z; walls in y
    (N, N, N, N, N, N),   # closed box (singular: pinned mode)
    (P, P, P, P, P, P),   # triply periodic (cyclic tridiagonal, singular mode)
    (D, N, P, P, N, D),
])
def test_homogeneous_faces_with_stretching(bc):
    n = (8, 16, 12)
    pts = [uniform_points(n[0]), geometric_points(n[1], 3.0), uniform_points(n[2])]
    if bc[2] == P:
        pts[1] = uniform_points(n[1])
    rng = np.random.default_rng(4)
    f = rng.standard_normal(n)
    if all(c in (N, P) for c in bc):
        V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
        f -= (f * V).sum() / V.sum()  # compatible right-hand side
    x = F.solve(f, pts, bc)
    r = F.laplacian_residual(x, f, pts, bc, (0.0,) * 6)
    assert np.abs(r).max() <= 1e-9


@pytest.mark.parametrize("bc,n", [
    ((P, P, D, D, P, P), (8, 16, 8)),   # channel with Dirichlet walls: periodic zero modes
    ((N, N, D, N, N, N), (8, 16, 4)),   # D-N solve direction, cosine zero modes
    ((N, N, D, D, N, N), (4, 8, 2)),    # D-D solve direction, tiny cosine transforms
])
def test_zero_transform_modes_are_regular_with_a_dirichlet_solve_direction(bc, n):
    """The mode whose two transform eigenvalues are zero is pinned only when
    the solve direction is N-N or periodic (tridiagonalSolver.C); with a
    Dirichlet face there the system is regular and the solution is the
    finite-volume system's, checked against a sparse direct solve of
    Laplacian(x) = -f built independently (tests/helpers.py)."""
    import scipy.sparse.linalg as spl

    from tests.helpers import brick_operator

    pts = [uniform_points(m) for m in n]
    pts[1] = geometric_points(n[1], 2.0)
    f = np.random.default_rng(3).standard_normal(n)
    x = F.solve(f, pts, bc)
    A, V, _ = brick_operator(pts, bc)
    xd = spl.spsolve(A.tocsc(), -(V.reshape(n) * f).ravel())
    assert np.linalg.norm(x.ravel() - xd) <= 1e-12 * np.linalg.norm(xd)


def test_known_answer_ddt():
    """Test-FFTPoissonSolverDdt.C: all faces Dirichlet 0, uniform mesh,
    random b and old x; Laplacian(x) - x/dt + b + x_old/dt = 0 per cell."""
    n = (16, 16, 16)
    pts = [uniform_points(m) for m in n]
    bc = (D,) * 6
    rng = np.random.default_rng(7)
    b = rng.random(n) - 0.5
    xo = rng.random(n) - 0.5
    dt = 0.01
    x = F.solve(b, pts, bc, shift=1.0 / dt, x_old=xo)
    r = F.laplacian_residual(x, b + xo / dt, pts, bc, (0.0,) * 6) - x / dt
    assert np.abs(r).max() <= 1e-10 * (1.0 / dt)


def test_shift_keeps_the_singular_mode_pin():
    """The reference pins the first diagonal entry of the mode whose two
    eigenvalues are zero (tridiagonalSolver.C:180-186, 225-231) whether or
    not a shift makes that mode regular; the restatement does the same, so
    a shifted solve on an all-Neumann/periodic box misses the equation at
    the first cell of the mean mode only."""
    n = (8, 8, 8)
    pts = [uniform_points(8), geometric_points(8, 2.0), uniform_points(8)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(5)
    f = rng.standard_normal(n)
    xo = rng.standard_normal(n)
    s = 7.5
    x = F.solve(f, pts, bc, shift=s, x_old=xo)
    r = F.laplacian_residual(x, f + s * xo, pts, bc, (0.0,) * 6) - s * x
    assert np.abs(r[:, 1:, :]).max() <= 1e-9
    # the residual at j = 0 is the same constant in every cell: the mean mode
    assert np.ptp(r[:, 0, :]) <= 1e-9 and abs(r[0, 0, 0]) > 1e-3


def _smooth_lambda(n, ratio, rng, periodic):
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


def test_split_divergence_is_the_laplacian_for_unit_lambda():
    n = (8, 12, 10)
    pts = [uniform_points(8), geometric_points(12, 2.0), uniform_points(10)]
    bc = (P, P, N, N, D, N)
    vals = (0.0, 0.0, 0.5, -0.3, 1.2, 0.7)
    x = np.random.default_rng(0).standard_normal(n)
    lam = [np.ones((9, 12, 10)), np.ones((8, 13, 10)), np.ones((8, 12, 11))]
    div = F.face_flux_divergence(x, lam, pts, bc, vals)
    assert np.abs(div - F.laplacian_residual(x, np.zeros(n), pts, bc, vals)).max() <= 1e-11


def test_split_converges_to_the_variable_coefficient_solution():
    """splitPoissonSolver.C:110-149: repeated corrections with the lagged
    variable part converge to -div(lambda grad x) = b (contraction factor
    about 1 - min lambda / max lambda)."""
    n = (16, 16, 16)
    pts = [uniform_points(16), geometric_points(16, 2.0), uniform_points(16)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(1)
    lam = _smooth_lambda(n, 1.5, rng, (True, False, True))
    b = rng.standard_normal(n)
    V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
    b -= (b * V).sum() / V.sum()
    res = [np.abs(F.variable_residual(F.split_solve(np.zeros(n), b, lam, pts, bc, n_corr=k), b, lam, pts, bc)).max()
           for k in (1, 5, 20)]
    assert res[0] > res[1] > res[2] and res[2] <= 1e-9


def test_projection_step_leaves_a_divergence_free_velocity():
    """briscolaStaggered.C:92-96 restated: p from coloDiv(U) / (-C dt), then
    U -= C dt stagReconstruct(faceGrad(p) A); the colocated divergence of the
    corrected velocity vanishes (the consistency of coloDiv, the solver's
    Laplacian and the reconstruction)."""
    n = (16, 24, 16)
    pts = [uniform_points(16), geometric_points(24, 2.0), uniform_points(16)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(0)
    u = [rng.standard_normal((17, 24, 16)), rng.standard_normal((16, 25, 16)), rng.standard_normal((16, 24, 17))]
    u[0][-1] = u[0][0]
    u[2][:, :, -1] = u[2][:, :, 0]
    u[1][:, 0, :] = 0.0  # no flux through the walls
    u[1][:, -1, :] = 0.0
    cdt = 0.05
    p = F.solve(F.colo_div(u, pts) / (-cdt), pts, bc)
    un = F.project_correct(u, p, cdt, pts, (True, False, True))
    assert np.abs(F.colo_div(u, pts)).max() > 10.0
    assert np.abs(F.colo_div(un, pts)).max() <= 1e-11
