"""Multi-brick solves on the GPU: one launch per level across all bricks, a
device-side ghost exchange between bricks, contacts expressed as face
lambdas.

* A brick split into pieces is the same discrete problem: the kernels give
  bit-identical results on the pieces and on the whole brick, and the
  solutions agree to rounding.
* The seven-brick layout (scaled down) matches a sparse direct FP64 solve
  of the union-domain operator to 1e-10.
* At full size (2.55 M cells) the FP64 and mixed solves reach 1e-8, checked
  with the union-domain operator on the host.
* Dirichlet faces and Neumann gradients on the bricks' wall faces
  (DirichletBoundaryCondition.C:19-80, NeumannBoundaryCondition.C:19-56,
  per brick face): split bricks are bit-identical to the whole brick, and an
  L-shaped three-brick domain matches the union-domain direct solve with the
  same wall conditions to 1e-10.
"""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import DIRICHLET, NEUMANN, PERIODIC, Brick, Mesh, geometric_points, uniform_points
from tests.helpers import (brick_to_compact, rel, split_brick, union_operator, union_operator_bc, union_solve,
                           vmean)

pytestmark = pytest.mark.gpu

# (brick, cuts): dyadic uniform coordinates keep every derived quantity exact
SPLITS = {
    "x2": (lambda: Brick([uniform_points(32)] * 3), ([16], [], [])),
    "y3": (lambda: Brick([uniform_points(32), uniform_points(32), uniform_points(16)]), ([], [8, 24], [])),
    "xyz8": (lambda: Brick([uniform_points(32)] * 3), ([16], [16], [16])),
    "graded_z": (lambda: Brick([uniform_points(16), geometric_points(16, 2.0), geometric_points(48, 0.5)]),
                 ([], [], [16, 32])),
    # periodic axes: the pieces meet across the box's periodic ends
    "periodic_x2": (lambda: Brick([uniform_points(32)] * 3, (PERIODIC, PERIODIC) + (NEUMANN,) * 4), ([16], [], [])),
    "channel_xz": (lambda: Brick([uniform_points(32), geometric_points(16, 2.0), uniform_points(32)],
                                 (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC)), ([16], [], [8, 24])),
    "periodic_spanning": (lambda: Brick([uniform_points(16), uniform_points(32), uniform_points(16)],
                                        (NEUMANN, NEUMANN, NEUMANN, NEUMANN, PERIODIC, PERIODIC)), ([8], [16], [])),
    # Dirichlet values and Neumann gradients on the wall faces (the pieces'
    # faces in contact are interfaces and drop the brick's conditions)
    "dirichlet_x2": (lambda: Brick([uniform_points(32)] * 3,
                                   (DIRICHLET, NEUMANN, NEUMANN, DIRICHLET, NEUMANN, NEUMANN),
                                   values=(1.0, 0.5, -0.25, 2.0, 0.0, 0.75)), ([16], [], [])),
    "dirichlet_xyz8_graded": (lambda: Brick([uniform_points(32), geometric_points(32, 2.0), uniform_points(32)],
                                            (DIRICHLET,) * 6, values=(1.0, -1.0, 0.5, 0.25, 2.0, -2.0)),
                              ([16], [16], [16])),
    "dirichlet_channel_xz": (lambda: Brick([uniform_points(32), geometric_points(16, 2.0), uniform_points(32)],
                                           (PERIODIC, PERIODIC, DIRICHLET, DIRICHLET, PERIODIC, PERIODIC),
                                           values=(0.0, 0.0, 1.0, -1.0, 0.0, 0.0)), ([16], [], [8, 24])),
}


def _ctx(mesh, **kw):
    d = {"autotune": "off", "relTol": 1e-12, "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2}
    d.update(kw)
    return bb.Context(mesh, bb.make_options(d))


def _whole_and_parts(name):
    mk, cuts = SPLITS[name]
    br = mk()
    return br, Mesh([br]), split_brick(br, cuts)


def _to_parts(parts, level, full, whole_shape):
    """whole-brick field of a level -> the pieces' compact order"""
    out = []
    for q, br in enumerate(parts.bricks):
        s = 2 ** level
        o = [br.origin[d] // s for d in range(3)]
        n = [br.N[d] // s for d in range(3)]
        out.append(full[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]].ravel())
    return np.concatenate(out)


@pytest.mark.parametrize("name", ["x2", "y3", "xyz8", "periodic_x2", "channel_xz", "periodic_spanning",
                                  "dirichlet_x2", "dirichlet_xyz8_graded", "dirichlet_channel_xz"])
@pytest.mark.parametrize("precision", [0, 1])
def test_split_building_blocks_bit_identical(native, name, precision):
    br, whole, parts = _whole_and_parts(name)
    cw = _ctx(whole, fused="off")
    cp = _ctx(parts)
    rng = np.random.default_rng(11)
    nlev = min(cw.num_levels, cp.num_levels)
    for l in range(nlev):
        shp = cw.shape(l)
        assert sum(int(np.prod(s)) for s in cp.shapes(l)) == int(np.prod(shp))
        x = rng.standard_normal(shp)
        b = rng.standard_normal(shp)
        for colour in (0, 1, 1, 0):
            cw.upload(l, "x", x, precision)
            cw.upload(l, "b", b, precision)
            cp.upload(l, "x", _to_parts(parts, l, x, shp), precision)
            cp.upload(l, "b", _to_parts(parts, l, b, shp), precision)
            cw.colour_pass(l, colour, precision)
            cp.colour_pass(l, colour, precision)
            assert np.array_equal(_to_parts(parts, l, cw.download(l, "x", precision), shp),
                                  cp.download(l, "x", precision)), (l, colour)
        assert np.array_equal(_to_parts(parts, l, cw.residual(l, precision), shp), cp.residual(l, precision))
        if l + 1 < nlev:
            # residual + restriction, then prolongation + correction
            cw.residual_restrict(l, precision)
            cp.residual_restrict(l, precision)
            cs = cw.shape(l + 1)
            assert np.array_equal(_to_parts(parts, l + 1, cw.download(l + 1, "b", precision), cs),
                                  cp.download(l + 1, "b", precision)), l
            xc = rng.standard_normal(cs)
            cw.upload(l + 1, "x", xc, precision)
            cp.upload(l + 1, "x", _to_parts(parts, l + 1, xc, cs), precision)
            cw.prolong_correct(l, precision)
            cp.prolong_correct(l, precision)
            assert np.array_equal(_to_parts(parts, l, cw.download(l, "x", precision), shp),
                                  cp.download(l, "x", precision)), l


@pytest.mark.parametrize("name", list(SPLITS))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_solve_matches_whole_brick(native, name, precision):
    br, whole, parts = _whole_and_parts(name)
    rng = np.random.default_rng(21)
    V = br.cell_volumes()
    f = rng.standard_normal(br.N)
    bfull = -V * (f - (V * f).sum() / V.sum())
    cp = _ctx(parts, precision=precision)
    lc = cp.coarse_level_index
    # the whole brick solves directly on the same level
    cw = _ctx(whole, precision=precision, coarseLevel=cw_levels(whole) - 1 - lc)
    assert cw.coarse_level_index == lc
    xw = np.zeros(br.N)
    rw = cw.solve(np.ascontiguousarray(bfull), xw, zero_guess=True)
    bp = brick_to_compact(parts, bfull)
    xp = np.zeros_like(bp)
    rp = cp.solve(bp, xp, zero_guess=True)
    assert rw.status == 0 and rp.status == 0
    assert abs(rw.cycles - rp.cycles) <= 1
    tol = 1e-10 if precision == "fp64" else 1e-8
    assert rel(xp, brick_to_compact(parts, xw)) <= tol


def cw_levels(mesh):
    return bb.Context(mesh, bb.make_options({"autotune": "off"})).num_levels


def test_split_variable_coefficient(native):
    br = Brick([uniform_points(32)] * 3)
    whole, parts = Mesh([br]), split_brick(br, ([16], [8], []))
    rng = np.random.default_rng(4)
    lam = [np.exp(rng.uniform(-2, 2, s)) for s in ((33, 32, 32), (32, 33, 32), (32, 32, 33))]
    lam_p = []
    for d in range(3):
        pieces = []
        for p in parts.bricks:
            o, n = p.origin, list(p.N)
            n[d] += 1
            pieces.append(lam[d][o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]].ravel())
        lam_p.append(np.concatenate(pieces))
    V = br.cell_volumes()
    f = rng.standard_normal(br.N)
    bfull = -V * (f - (V * f).sum() / V.sum())
    cp = _ctx(parts)
    cw = _ctx(whole, coarseLevel=cw_levels(whole) - 1 - cp.coarse_level_index)
    cw.set_coefficients(lam)
    cp.set_coefficients(lam_p)
    xw = np.zeros(br.N)
    assert cw.solve(np.ascontiguousarray(bfull), xw, zero_guess=True).status == 0
    bp = brick_to_compact(parts, bfull)
    xp = np.zeros_like(bp)
    assert cp.solve(bp, xp, zero_guess=True).status == 0
    assert rel(xp, brick_to_compact(parts, xw)) <= 1e-10


@pytest.mark.parametrize("scale", [4, 8])
def test_multibrick_matches_union_direct_solve(native, scale):
    mesh, b, _ = workloads.multibrick(scale)
    xref, V = union_solve(mesh, b)
    c = _ctx(mesh, relTol=1e-13, maxIter=200)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    assert rel(x, xref) <= 1e-10


@pytest.mark.parametrize("cyc,smoother", [("W", "rbgs"), ("F", "rbgs"), ("V", "jac")])
def test_multibrick_cycles_and_smoothers(native, cyc, smoother):
    mesh, b, _ = workloads.multibrick(4)
    xref, V = union_solve(mesh, b)
    c = _ctx(mesh, relTol=1e-10, maxIter=400, cycleType=cyc, smoother=smoother)
    x = np.zeros_like(b)
    assert c.solve(b, x, zero_guess=True).status == 0
    assert rel(x, xref) <= 1e-7


def test_multibrick_graph_matches_host_loop(native):
    mesh, b, _ = workloads.multibrick(4)
    xs = {}
    for g in ("on", "off"):
        c = _ctx(mesh, graph=g, relTol=1e-10)
        x = np.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        assert rep.status == 0
        xs[g] = (x, rep.cycles)
    assert xs["on"][1] == xs["off"][1] and np.array_equal(xs["on"][0], xs["off"][0])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multibrick_full_size(native, precision):
    mesh, b, _ = workloads.multibrick(1)
    A, V = union_operator(mesh)
    c = _ctx(mesh, relTol=1e-8, precision=precision, autotune="on")
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    r = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    # the device's FP64 residual is the host's
    assert abs(r - rep.rel_residual) <= 1e-6 * r + 1e-15
    assert rep.final_residual <= 1e-8 * rep.initial_residual
    assert abs((V * x).sum()) <= 1e-12 * np.abs(V * x).sum()


def _l_shape():
    """Three 32 x 32 x 16 bricks in an L (cells of 1/64): A at the corner, B
    beyond A along x, C beyond A along y; A-B and A-C share whole faces.
    Dirichlet values on A's and C's x-lo, B's x-hi and y-lo and C's y-hi,
    Neumann gradients on C's x-hi and A's z-lo, zero-gradient walls
    elsewhere."""
    h = 1 / 64

    def pts(n, o):
        return (o + np.arange(n + 1)) * h

    D, N = DIRICHLET, NEUMANN
    A = Brick([pts(32, 0), pts(32, 0), pts(16, 0)], (D, N, N, N, N, N), (0, 0, 0), (1.0, 0, 0, 0, 0.1, 0))
    B = Brick([pts(32, 32), pts(32, 0), pts(16, 0)], (N, D, D, N, N, N), (32, 0, 0), (0, -0.5, 0.25, 0, 0, 0))
    C = Brick([pts(32, 0), pts(32, 32), pts(16, 0)], (D, N, N, D, N, N), (0, 32, 0), (1.0, 0.3, 0, -1.0, 0, 0))
    return Mesh([A, B, C])


def test_multibrick_dirichlet_matches_union_direct_solve(native):
    import scipy.sparse.linalg as spl

    mesh = _l_shape()
    A, V, bdir = union_operator_bc(mesh)
    rng = np.random.default_rng(31)
    b = -V * rng.standard_normal(V.size)
    xref = spl.spsolve(A.tocsc(), b + bdir)
    c = _ctx(mesh, relTol=1e-13, maxIter=200)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    assert rel(x, xref) <= 1e-10
    # the mixed solve with flexible CG, on the true residual of the union operator
    c = _ctx(mesh, relTol=1e-10, precision="mixed", krylov="fcg", maxIter=100)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    beff = b + bdir
    assert np.linalg.norm(A @ x - beff) <= 2e-10 * np.linalg.norm(beff)
