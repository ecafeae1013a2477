"""Pins of the CPU oracle (no GPU).

The reference has no golden vectors for its multigrid; what pins the path
are its known-answer tests, restated here on the oracle:
  * restriction exactness for constant and linear fields, <= 1e-14
    (applications/test/restriction/Test-restriction.C:15-194, mesh 32x64x96);
  * prolongation exactness with ghost values set to the exact field, <= 1e-14
    (applications/test/prolongation/Test-prolongation.C:15-110);
  * the pointwise discrete-Laplacian residual <= 1e-10 on geometrically
    graded meshes (applications/test/FFTPoissonSolver/Test-FFTPoissonSolver.C
    :11-92, stretch set of run.sh; homogeneous Neumann walls here).
Independent FP64 ground truths (DCT, FFT + Thomas, sparse direct) pin the
converged solutions.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from briscola_b200 import workloads
from briscola_b200.mesh import geometric_points
from oracle.pyoracle import Oracle
from tests.helpers import channel_solution, dct_neumann_solution, rel, uniform, vmean

V22 = dict(n_pre=2, n_post=2, cycle_type="V", coarse_level=1)


def _grids(o, l):
    cx, cy, cz = (o.centres(l, d) for d in range(3))
    return cx, cy, cz


@pytest.mark.parametrize("stretch", [(1, 1, 1), (2, 1, 1), (1, 1, 2)])
def test_restriction_known_answer(stretch):
    N = (32, 64, 96)
    pts = [geometric_points(N[d], stretch[d]) for d in range(3)]
    o = Oracle(pts, nthreads=2)
    fields = {
        "const": lambda x, y, z: 2.0 + 0 * x,
        "x": lambda x, y, z: x, "y": lambda x, y, z: y, "z": lambda x, y, z: z,
        "xy": lambda x, y, z: x + y, "xz": lambda x, y, z: x + z, "yz": lambda x, y, z: y + z,
        "xyz": lambda x, y, z: x + y + z,
    }
    for name, f in fields.items():
        cx, cy, cz = _grids(o, 0)
        fl = f(cx[1:-1, None, None], cy[None, 1:-1, None], cz[None, None, 1:-1]) * np.ones(o.shape(0))
        for l in range(o.num_levels - 1):
            fl = o.restrict(l, fl, scale=False)
            cx, cy, cz = _grids(o, l + 1)
            exact = f(cx[1:-1, None, None], cy[None, 1:-1, None], cz[None, None, 1:-1]) * np.ones(o.shape(l + 1))
            assert np.max(np.abs(fl - exact)) <= 1e-14, (name, l)


@pytest.mark.parametrize("stretch", [(1, 1, 1), (1, 2, 1)])
def test_prolongation_known_answer(stretch):
    N = (32, 64, 96)
    pts = [geometric_points(N[d], stretch[d]) for d in range(3)]
    o = Oracle(pts, nthreads=2)
    for name, f in {"const": lambda x, y, z: 2.0 + 0 * x, "x": lambda x, y, z: x, "y": lambda x, y, z: y,
                    "z": lambda x, y, z: z, "xyz": lambda x, y, z: x + y + z}.items():
        for l in range(o.num_levels - 1, 0, -1):
            cx, cy, cz = _grids(o, l)
            coarse_g = f(cx[:, None, None], cy[None, :, None], cz[None, None, :]) * np.ones(
                tuple(n + 2 for n in o.shape(l)))
            fine = o.prolong_ghosted(l - 1, coarse_g, op="=")
            fx, fy, fz = _grids(o, l - 1)
            exact = f(fx[1:-1, None, None], fy[None, 1:-1, None], fz[None, None, 1:-1]) * np.ones(o.shape(l - 1))
            assert np.max(np.abs(fine - exact)) <= 1e-14, (name, l)


@pytest.mark.parametrize("stretch", [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2)])
def test_laplacian_pointwise_known_answer(stretch):
    N = (16, 64, 32)
    pts = [geometric_points(N[d], stretch[d]) for d in range(3)]
    o = Oracle(pts, nthreads=2)
    rng = np.random.default_rng(123)
    f = 100.0 * rng.random(N) - 0.5
    dx, dy, dz = (np.diff(p) for p in pts)
    V = dx[:, None, None] * dy[None, :, None] * dz[None, None, :]
    f = f - (V * f).sum() / V.sum()
    b = -V * f
    # cells of aspect ratio 4 slow point-smoothed multigrid down: many cycles
    p, rep, _, rc = o.solve(b, rel_tol=1e-14, max_iter=600, **V22)
    # Test-FFTPoissonSolver.C:11-92 with zero-gradient ghosts
    pg = np.pad(p, 1, mode="edge")
    def d2(axis, h):
        hp = np.pad(h, 1, mode="edge")
        hw = 0.5 * (hp[1:-1] + hp[:-2])
        he = 0.5 * (hp[1:-1] + hp[2:])
        sl = [None, None, None]
        sl[axis] = slice(None)
        hw, he, hh = hw[tuple(sl)], he[tuple(sl)], h[tuple(sl)]
        c = pg[1:-1, 1:-1, 1:-1]
        m = [slice(1, -1)] * 3
        q = [slice(1, -1)] * 3
        m[axis] = slice(0, -2)
        q[axis] = slice(2, None)
        return pg[tuple(m)] / (hw * hh) - c / (hw * hh) - c / (he * hh) + pg[tuple(q)] / (he * hh)
    res = d2(0, dx) + d2(1, dy) + d2(2, dz) + f
    assert np.max(np.abs(res)) <= 1e-10, np.max(np.abs(res))


def test_dct_ground_truth():
    mesh, b, _ = workloads.cavity(32, seed=7)
    br = mesh.bricks[0]
    o = Oracle(br.points, nthreads=2)
    x, rep, hist, rc = o.solve(b.reshape(br.N), rel_tol=1e-13, max_iter=100, **V22)
    assert rc == 0
    xt = dct_neumann_solution(b.reshape(br.N), 1.0 / 32)
    V = br.cell_volumes()
    assert rel(vmean(x, V), vmean(xt, V)) <= 1e-10


def test_channel_ground_truth():
    mesh, b, _ = workloads.channel(32, seed=9)
    br = mesh.bricks[0]
    o = Oracle(br.points, periodic=br.periodic, nthreads=2)
    x, rep, hist, rc = o.solve(b.reshape(br.N), rel_tol=1e-13, max_iter=100, **V22)
    assert rc == 0
    xt = channel_solution(b.reshape(br.N), *br.points)
    V = br.cell_volumes()
    assert rel(vmean(x, V), vmean(xt, V)) <= 1e-10


def _sparse_from_oracle(o, l=0):
    A7 = o.matrix(l)
    n0, n1, n2 = o.shape(l)
    idx = np.arange(n0 * n1 * n2).reshape(n0, n1, n2)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [A7[..., 0].ravel()]
    for s, (ax, sh) in enumerate([(0, -1), (0, 1), (1, -1), (1, 1), (2, -1), (2, 1)], start=1):
        nb = np.roll(idx, -sh, axis=ax)
        rows.append(idx.ravel())
        cols.append(nb.ravel())
        vals.append(A7[..., s].ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(idx.size, idx.size))
    A.eliminate_zeros()
    return A


def test_variable_coefficient_against_sparse_direct():
    mesh, b, lam = workloads.sphere(16, seed=11)
    br = mesh.bricks[0]
    o = Oracle(br.points, nthreads=2)
    o.set_lambda(*lam)
    x, rep, hist, rc = o.solve(b.reshape(br.N), rel_tol=1e-13, max_iter=200, **V22)
    assert rc == 0
    o.assemble(**V22)
    A = _sparse_from_oracle(o).tolil()
    A[0, :] = 0
    A[0, 0] = 1.0  # pin for the direct solve (the RHS is compatible)
    rhs = b.copy()
    rhs[0] = 0.0
    xt = spla.spsolve(A.tocsr(), rhs).reshape(br.N)
    V = br.cell_volumes()
    assert rel(vmean(x, V), vmean(xt, V)) <= 1e-9


def test_area_weighted_lambda_restriction_constant():
    br_pts = [uniform(8), geometric_points(16, 2.0), uniform(8)]
    o = Oracle(br_pts, nthreads=1)
    lam = [np.full((9, 16, 8), 3.0), np.full((8, 17, 8), 3.0), np.full((8, 16, 9), 3.0)]
    o.set_lambda(*lam)
    for l in range(o.num_levels):
        for fd in range(3):
            assert np.allclose(o.get_lambda(l, fd), 3.0, rtol=0, atol=1e-14)


def test_reference_sweep_equals_colour_sequence():
    """On an all-wall brick one reference RBGS sweep (four loop-counter passes,
    rbgsSmoother.C:65-183) is the colour sequence 0, 1, q, 1-q with
    q = (n0+n1+n2+1) % 2 -- the order the GPU smoother applies."""
    for N in [(8, 8, 8), (8, 6, 4), (6, 5, 4), (3, 4, 5)]:
        o = Oracle([uniform(n) for n in N], nthreads=1)
        o.assemble(**V22)
        rng = np.random.default_rng(3)
        x0 = rng.standard_normal(N)
        b = rng.standard_normal(N)
        ref = o.smooth(0, x0, b, sweeps=2)
        q = (sum(N) + 1) % 2
        seq = []
        for _ in range(2):
            for c in (0, 1, q, 1 - q):
                if not seq or seq[-1] != c:
                    seq.append(c)
        x = x0.copy()
        for c in seq:
            x = o.colour_pass(0, c, x, b)
        assert np.array_equal(ref, x), N


@pytest.mark.parametrize("cyc", ["V", "W", "F"])
@pytest.mark.parametrize("smoother", ["rbgs", "jac"])
def test_oracle_cycles_converge(cyc, smoother):
    mesh, b, _ = workloads.cavity(16, seed=5)
    br = mesh.bricks[0]
    o = Oracle(br.points, nthreads=1)
    x, rep, hist, rc = o.solve(b.reshape(br.N), rel_tol=1e-10, max_iter=200, n_pre=2, n_post=2,
                               cycle_type=cyc, coarse_level=1, smoother=smoother)
    assert rc == 0 and rep.final_residual / rep.initial_residual <= 1e-10


def test_thread_count_does_not_change_results():
    mesh, b, _ = workloads.channel(32, seed=3)
    br = mesh.bricks[0]
    outs = []
    for nt in (1, 4):
        o = Oracle(br.points, periodic=br.periodic, nthreads=nt)
        x, rep, hist, rc = o.solve(b.reshape(br.N), rel_tol=1e-8, **V22)
        outs.append((x, rep.iterations))
    assert outs[0][1] == outs[1][1]
    assert np.array_equal(outs[0][0], outs[1][0])
