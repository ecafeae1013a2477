"""Brick orientations on the GPU (bmg_brick.transform, the role of the
transform T of parallelBoundaryCondition.C:148-163): a mesh whose bricks are
described in rotated and reflected frames is the same discrete problem as the
axis-aligned one.  The device keeps every brick in the mesh's frame and reads
and writes the caller's arrays (b, x, lambda) in each brick's frame, so the
solutions agree bit for bit once mapped back."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200.mesh import Brick, Mesh, geometric_points, uniform_points
from tests.helpers import split_brick
from tests.orient import lambda_to_local, orient, to_local, to_mesh

pytestmark = pytest.mark.gpu

T = [(0, 0, 0), (2, -1, 3), (-3, 2, -1), (-1, -2, -3), (3, 1, 2), (-2, 3, 1), (1, -3, 2), (3, -2, -1)]


def _ctx(mesh, **kw):
    d = {"autotune": "off", "relTol": 1e-12, "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2,
         "maxIter": 100}
    d.update(kw)
    return bb.Context(mesh, bb.make_options(d))


def _lam(n, rng):
    out = []
    for d in range(3):
        shape = list(n)
        shape[d] += 1
        out.append(np.exp(rng.uniform(-1.0, 1.0, shape)))
    return out


def _solve_pair(parts, transforms, b_mesh, lam_mesh, **kw):
    """solve the axis-aligned parts and the oriented parts; return both
    solutions per brick in the mesh frame"""
    bricks = parts.bricks
    oriented = Mesh([orient(br, transforms[q]) for q, br in enumerate(bricks)])
    out = []
    for mesh, ts in ((parts, [(0, 0, 0)] * len(bricks)), (oriented, transforms)):
        c = _ctx(mesh, **kw)
        if lam_mesh is not None:
            lams = [lambda_to_local(lam_mesh[q], ts[q]) for q in range(len(bricks))]
            c.set_coefficients([np.concatenate([l[d].ravel() for l in lams]) for d in range(3)])
        b = np.concatenate([to_local(b_mesh[q], ts[q]).ravel() for q in range(len(bricks))])
        x = np.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        assert rep.status == 0, (ts, rep.status, rep.cycles, rep.final_residual / max(rep.initial_residual, 1e-300))
        xs, o = [], 0
        for q, br in enumerate(mesh.bricks):
            n = br.N
            xs.append(to_mesh(x[o:o + int(np.prod(n))].reshape(n), ts[q]))
            o += int(np.prod(n))
        out.append((xs, rep))
        c.close()
    return out


@pytest.mark.parametrize("precision,krylov", [("fp64", "none"), ("mixed", "fcg")])
@pytest.mark.parametrize("variable", [False, True])
def test_oriented_bricks_reproduce_the_aligned_solve(native, precision, krylov, variable):
    whole = Brick([uniform_points(32), geometric_points(16, 2.0), geometric_points(48, 0.5)])
    parts = split_brick(whole, ([16], [], [16, 32]))
    rng = np.random.default_rng(3)
    b = [rng.standard_normal(br.N) for br in parts.bricks]
    # a compatible system right-hand side (b_sys = -V f sums to zero)
    total = sum(x.sum() for x in b)
    ncell = sum(x.size for x in b)
    b = [x - total / ncell for x in b]
    lam = [_lam(br.N, rng) for br in parts.bricks] if variable else None
    if lam is not None:  # a face shared by two bricks carries one value
        for q, br in enumerate(parts.bricks):
            for r, other in enumerate(parts.bricks):
                for d in range(3):
                    if other.origin[d] == br.origin[d] + br.N[d] and all(
                            other.origin[e] == br.origin[e] for e in range(3) if e != d):
                        hi = [slice(None)] * 3
                        lo = [slice(None)] * 3
                        hi[d], lo[d] = -1, 0
                        lam[r][d][tuple(lo)] = lam[q][d][tuple(hi)]
    transforms = T[1:1 + len(parts.bricks)]
    (xa, ra), (xo, ro) = _solve_pair(parts, transforms, b, lam, precision=precision, krylov=krylov)
    assert ra.cycles == ro.cycles
    for p, q in zip(xa, xo):
        assert np.array_equal(p, q)


@pytest.mark.parametrize("t", T[1:])
def test_oriented_single_brick_with_walls_and_values(native, t):
    br = Brick([uniform_points(32), geometric_points(16, 2.0), uniform_points(16)],
               ("Dirichlet", "Neumann", "Neumann", "Dirichlet", "periodic", "periodic"),
               values=(1.0, 0.3, 0.0, -2.0, 0.0, 0.0))
    rng = np.random.default_rng(4)
    b = [rng.standard_normal(br.N)]
    lam = [_lam(br.N, rng)]
    for d in (2,):  # periodic axis: the last face repeats the first
        lam[0][d][:, :, -1] = lam[0][d][:, :, 0]
    (xa, ra), (xo, ro) = _solve_pair(Mesh([br]), [t], b, lam, precision="mixed", krylov="fcg")
    assert ra.cycles == ro.cycles
    assert np.array_equal(xa[0], xo[0])


def test_level_shapes_are_in_the_brick_frame(native):
    br = orient(Brick([uniform_points(32), uniform_points(16), uniform_points(8)]), (3, -1, 2))
    c = _ctx(Mesh([br]))
    assert c.shape(0) == (8, 32, 16)
    assert c.shape(1) == (4, 16, 8)
    x = np.random.default_rng(5).standard_normal(c.shape(1))
    c.upload(1, "x", x)
    assert np.array_equal(c.download(1, "x"), x)
    c.close()
