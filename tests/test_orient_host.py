"""Brick orientations on the host: the test helpers' frame changes are
inverse to each other and move face arrays with their faces, and
bmg_create checks a transform before it touches a device."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200.mesh import Brick, Mesh, geometric_points, uniform_points
from tests.orient import lambda_to_local, orient, to_local, to_mesh

TRANSFORMS = [(2, -1, 3), (-3, 2, -1), (-1, -2, -3), (3, 1, 2)]


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except ImportError:
        return True


@pytest.mark.parametrize("t", TRANSFORMS)
def test_frame_changes_are_inverse(t):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((4, 5, 6))
    loc = to_local(a, t)
    tax = [abs(v) - 1 for v in t]
    assert loc.shape == tuple(a.shape[tax[d]] for d in range(3))
    assert np.array_equal(to_mesh(loc, t), a)
    # a face array keeps its face axis
    lam = [rng.standard_normal((5, 5, 6)), rng.standard_normal((4, 6, 6)), rng.standard_normal((4, 5, 7))]
    ll = lambda_to_local(lam, t)
    for ld in range(3):
        shape = [a.shape[tax[d]] + (d == ld) for d in range(3)]
        assert ll[ld].shape == tuple(shape)


def test_oriented_brick_keeps_its_geometry():
    br = Brick([uniform_points(8), geometric_points(6, 2.0), geometric_points(4, 0.5)],
               ("Dirichlet", "Neumann", "periodic", "periodic", "Neumann", "Neumann"),
               values=(1.0, 0.5, 0.0, 0.0, -0.25, 0.0))
    for t in TRANSFORMS:
        ob = orient(br, t)
        assert np.allclose(to_mesh(ob.cell_volumes(), t), br.cell_volumes(), rtol=1e-15)
        tax = [abs(v) - 1 for v in t]
        for d in range(3):
            assert ob.bc[2 * d] == br.bc[2 * tax[d] + (1 if t[d] < 0 else 0)]


def _create_error(mesh):
    with pytest.raises(bb.FatalError) as e:
        bb.Context(mesh, bb.make_options({}))
    return str(e.value)


@pytest.mark.parametrize("t", [(1, 1, 3), (4, 2, 1), (0, 2, 3), (-2, 2, 3)])
def test_invalid_transform_is_rejected(t):
    br = Brick([uniform_points(8)] * 3, transform=t)
    assert "invalid argument" in _create_error(Mesh([br]))


def test_reversed_axis_needs_decreasing_points():
    br = Brick([uniform_points(8)] * 3, transform=(-1, 2, 3))  # increasing points on a reversed axis
    assert "invalid argument" in _create_error(Mesh([br]))


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_valid_oriented_mesh_passes_the_host_checks():
    from tests.helpers import split_brick

    whole = Brick([uniform_points(16), uniform_points(8), uniform_points(24)])
    parts = split_brick(whole, ([8], [], [8]))
    m = Mesh([orient(b, TRANSFORMS[q % 4]) for q, b in enumerate(parts.bricks)])
    assert "no usable" in _create_error(m)
