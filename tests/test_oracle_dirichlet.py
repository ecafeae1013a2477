"""Dirichlet walls in the CPU restatement of the multigrid solve
(oracle/bmg_oracle.cpp: DirichletBoundaryCondition.C:19-80, the singularity
test of linearSystem.H:227-230) against an independent sparse direct solve
of the same finite-volume system (tests/helpers.py brick_operator): mixed
Dirichlet / Neumann / periodic faces, inhomogeneous values, stretched axes
and a variable coefficient; the eliminated matrix, the ghost rule the
prolongation reads and the unpinned coarse solve."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle, _dp, lib
from tests.helpers import brick_operator, rel

D, N, P = "Dirichlet", "Neumann", "periodic"

CASES = [
    ((D, D, D, D, D, D), (0.0,) * 6),
    ((D, N, N, N, N, N), (1.5, 0, 0, 0, 0, 0)),       # one outflow-like face
    ((N, D, P, P, D, N), (0, -0.5, 0, 0, 2.0, 0)),    # periodic y, mixed walls
    ((P, P, D, D, P, P), (0, 0, 1.0, -1.0, 0, 0)),    # channel with set wall values
    ((D, N, N, N, N, N), (1.5, 0.7, -0.3, 0, 0, 0.2)),  # Neumann gradients beside a Dirichlet face
]


def geometry(periodic):
    from briscola_b200.mesh import geometric_points, uniform_points

    return [uniform_points(16), geometric_points(8, 2.0) if not periodic[1] else uniform_points(8),
            geometric_points(12, 0.5) if not periodic[2] else uniform_points(12)]


def lam_field(n, rng, periodic):
    lam = []
    for d in range(3):
        shape = list(n)
        shape[d] += 1
        a = 0.5 + rng.random(shape)
        if periodic[d]:
            first = [slice(None)] * 3
            last = [slice(None)] * 3
            first[d], last[d] = 0, -1
            a[tuple(last)] = a[tuple(first)]
        lam.append(a)
    return lam


@pytest.mark.parametrize("bc,values", CASES)
@pytest.mark.parametrize("variable", [False, True])
def test_solution_matches_a_sparse_direct_solve(bc, values, variable):
    import scipy.sparse.linalg as spl

    periodic = tuple(bc[2 * d] == P for d in range(3))
    pts = geometry(periodic)
    n = tuple(len(p) - 1 for p in pts)
    rng = np.random.default_rng(7)
    lam = lam_field(n, rng, periodic) if variable else None
    A, V, bdir = brick_operator(pts, bc, values, lam)
    b = rng.standard_normal(int(np.prod(n)))
    ref = spl.spsolve(A.tocsc(), b + bdir)
    o = Oracle(pts, periodic, nthreads=4, dirichlet=[f == D for f in bc], values=values)
    if variable:
        o.set_lambda(*lam)
    x, rep, hist, rc = o.solve(b.reshape(n), rel_tol=1e-13, cycle_type="V", n_pre=2, n_post=2,
                               coarse_level=1, max_iter=200)
    assert rc == 0
    assert rel(x.ravel(), ref) <= 1e-10
    assert rep.iterations < 40


def test_eliminated_matrix_and_no_pin():
    pts = geometry((False, False, False))
    bc = (D, N, N, D, N, N)
    o = Oracle(pts, dirichlet=[f == D for f in bc])
    o.assemble(coarse_level=0)
    A0 = o.matrix(0)
    Asp, V, _ = brick_operator(pts, bc)
    n = A0.shape[:3]
    dense = Asp.toarray()
    assert np.allclose(A0[..., 0].ravel(), np.diag(dense), rtol=1e-14, atol=0)
    # every wall coupling dropped
    assert np.all(A0[0, :, :, 1] == 0) and np.all(A0[-1, :, :, 2] == 0)
    assert np.all(A0[:, 0, :, 3] == 0) and np.all(A0[:, -1, :, 4] == 0)
    # the coarsest level keeps its first row: no singularity pin
    L = o.num_levels - 1
    Ac = o.matrix(L)
    assert Ac[0, 0, 0, 0] != 1.0 and np.any(Ac[0, 0, 0, 1:] != 0)
    # and without a Dirichlet face the pin is there
    o2 = Oracle(pts)
    o2.assemble(coarse_level=0)
    assert o2.matrix(L)[0, 0, 0, 0] == 1.0


def test_prolongation_reads_the_mirrored_coarse_ghosts():
    """Coarse ghosts are -x at a Dirichlet wall on levels above 0
    (DirichletBoundaryCondition.C:59-80 with H = 0), a copy at a Neumann wall,
    and where two walls meet the unset-boundary copy of the diagonal interior
    cell (meshLevel.C:301-328)."""
    from briscola_b200.mesh import uniform_points

    pts = [uniform_points(8), uniform_points(8), uniform_points(8)]
    bc = (D, N, N, N, N, N)
    o = Oracle(pts, dirichlet=[f == D for f in bc])
    rng = np.random.default_rng(3)
    xc = rng.standard_normal(o.shape(1))
    out = np.zeros(o.shape(0))
    lib().bmgo_prolong(o._p, 0, _dp(np.ascontiguousarray(xc)), _dp(out), 0)
    # explicit ghosted array with the reference's rule
    g = np.zeros(tuple(s + 2 for s in xc.shape))
    g[1:-1, 1:-1, 1:-1] = xc
    g[0, 1:-1, 1:-1] = -xc[0]
    g[-1, 1:-1, 1:-1] = xc[-1]
    for d in (1, 2):
        lo = [slice(None)] * 3
        src = [slice(None)] * 3
        lo[d], src[d] = 0, 1
        g[tuple(lo)] = g[tuple(src)]
        lo[d], src[d] = -1, -2
        g[tuple(lo)] = g[tuple(src)]
    # wall-only edges and corners: copies of the diagonal interior cell
    n = xc.shape
    for i in range(-1, n[0] + 1):
        for j in range(-1, n[1] + 1):
            for k in range(-1, n[2] + 1):
                q = (i, j, k)
                out_axes = sum(v < 0 or v >= n[a] for a, v in enumerate(q))
                if out_axes >= 2:
                    c = tuple(min(max(v, 0), n[a] - 1) for a, v in enumerate(q))
                    g[i + 1, j + 1, k + 1] = xc[c]
    ref = np.zeros(o.shape(0))
    lib().bmgo_prolong_ghosted(o._p, 0, _dp(np.ascontiguousarray(g)), _dp(ref), 0)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("bc,values", [
    ((D, N, P, P, N, D), (1.0, 0.5, 0.0, 0.0, -0.25, 2.0)),
    ((N, D, N, N, P, P), (0.3, -1.0, 0.2, -0.4, 0.0, 0.0)),
])
def test_face_value_conventions_match_the_fft_restatement(bc, values):
    """The multigrid's face values (Dirichlet value, Neumann gradient) mean
    what the FFT solver's do (FFTPoissonSolver.C, oracle/fft_oracle.py): the
    same finite-volume system, so the split solver can hand one problem to
    both.  MG system A x = -V f + face terms; FFT: Laplacian(x) = -f."""
    import scipy.sparse.linalg as spl

    from briscola_b200.mesh import geometric_points, uniform_points
    from oracle import fft_oracle as F

    pts = [uniform_points(16), uniform_points(8), geometric_points(12, 2.0)]
    if bc[4] == P:
        pts[2] = uniform_points(12)
    n = tuple(len(p) - 1 for p in pts)
    f = np.random.default_rng(2).standard_normal(n)
    x_fft = F.solve(f, pts, bc, values)
    A, V, bdir = brick_operator(pts, bc, values)
    x_mg = spl.spsolve(A.tocsc(), -(V * f.ravel()) + bdir)
    assert rel(x_mg, x_fft.ravel()) <= 1e-10


@pytest.mark.parametrize("cycle", ["V", "W", "F"])
@pytest.mark.parametrize("options", [dict(), dict(coarse_direct=0), dict(restrict_average=1, prolong_injection=1)])
def test_every_cycle_option_reaches_the_direct_solution(cycle, options):
    """Cycle type, coarse mode and transfer schemes change how the oracle gets
    there, not where it goes: each reaches the sparse direct solution."""
    import scipy.sparse.linalg as spl

    bc, values = (D, N, P, P, N, D), (1.0, 0.0, 0.0, 0.0, 0.5, -1.0)
    periodic = (False, True, False)
    pts = geometry(periodic)
    n = tuple(len(p) - 1 for p in pts)
    A, V, bdir = brick_operator(pts, bc, values)
    b = np.random.default_rng(11).standard_normal(int(np.prod(n)))
    ref = spl.spsolve(A.tocsc(), b + bdir)
    o = Oracle(pts, periodic, nthreads=2, dirichlet=[f == D for f in bc], values=values)
    x, rep, hist, rc = o.solve(b.reshape(n), rel_tol=1e-12, cycle_type=cycle, n_pre=2, n_post=2, coarse_level=1,
                               max_iter=400, **options)
    assert rc == 0
    assert rel(x.ravel(), ref) <= 1e-9
