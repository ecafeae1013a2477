"""Multi-brick meshes on the host: the seven-brick workload's layout, the
union-domain operator used as ground truth by the GPU tests, and the mesh
checks bmg_create makes before it touches a device."""
import numpy as np
import pytest
import scipy.sparse.csgraph as csg

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import PERIODIC, Brick, Mesh, geometric_points, uniform_points
from tests.helpers import brick_to_compact, split_brick, union_operator, union_solve


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except ImportError:
        return True


def test_multibrick_layout():
    mesh, b, _ = workloads.multibrick(1)
    sizes = sorted(br.N for br in mesh.bricks)
    assert sizes == sorted(n for n, _ in workloads.MULTIBRICK_LAYOUT)
    assert mesh.n_cells == 2547712 and b.size == mesh.n_cells
    assert abs(b.sum()) <= 1e-12 * np.abs(b).sum()
    for br in mesh.bricks:
        assert all(o % 16 == 0 for o in br.origin)
        assert np.allclose(np.diff(br.points[0]), 1 / 128)


@pytest.mark.parametrize("scale", [2, 4, 8])
def test_multibrick_union_is_connected_neumann(scale):
    mesh, b, _ = workloads.multibrick(scale)
    A, V = union_operator(mesh)
    assert A.shape[0] == mesh.n_cells
    assert abs(A - A.T).max() < 1e-15
    assert np.abs(np.asarray(A.sum(axis=1))).max() < 1e-13
    ncomp, _ = csg.connected_components(A, directed=False)
    assert ncomp == 1  # one pin fixes the null space


def test_union_operator_of_split_brick_is_the_brick_operator():
    br = Brick([geometric_points(12, 2.0), uniform_points(8), uniform_points(10)])
    whole = Mesh([br])
    parts = split_brick(br, ([4, 8], [6], []))
    A1, _ = union_operator(whole)
    A2, _ = union_operator(parts)
    perm = brick_to_compact(parts, np.arange(12 * 8 * 10).reshape(12, 8, 10))
    assert abs(A1[perm][:, perm] - A2).max() < 1e-15


def test_union_solve_small():
    mesh, b, _ = workloads.multibrick(8)
    x, V = union_solve(mesh, b)
    A, _ = union_operator(mesh)
    assert np.linalg.norm(A @ x - b) <= 1e-12 * np.linalg.norm(b)
    assert abs((V * x).sum()) < 1e-12 * np.abs(x).sum()


def _create_error(mesh):
    with pytest.raises(bb.FatalError) as e:
        bb.Context(mesh, bb.make_options({}))
    return str(e.value)


def _pts(n, o, h=1 / 16):
    return o * h + h * np.arange(n + 1, dtype=np.float64)


def test_overlapping_bricks_are_rejected():
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], origin=(0, 0, 0)),
              Brick([_pts(8, 4), _pts(8, 0), _pts(8, 0)], origin=(4, 0, 0))])
    assert "invalid argument" in _create_error(m)


def test_mismatched_contact_coordinates_are_rejected():
    a = Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], origin=(0, 0, 0))
    b = Brick([_pts(8, 8) + 0.01, _pts(8, 0), _pts(8, 0)], origin=(8, 0, 0))
    assert "invalid argument" in _create_error(Mesh([a, b]))
    # tangential coordinates must match too
    c = Brick([_pts(8, 8), _pts(8, 0) * 1.1, _pts(8, 0)], origin=(8, 0, 0))
    assert "invalid argument" in _create_error(Mesh([a, c]))


def test_periodic_axis_must_be_periodic_for_every_brick():
    bc = (PERIODIC, PERIODIC) + ("Neumann",) * 4
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], bc, (0, 0, 0)),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], ("Neumann",) * 6, (0, 8, 0))])
    assert "invalid argument" in _create_error(m)


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_periodic_multibrick_passes_the_host_checks():
    bc = (PERIODIC, PERIODIC) + ("Neumann",) * 4
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], bc, (0, 0, 0)),
              Brick([_pts(8, 8), _pts(8, 0), _pts(8, 0)], bc, (8, 0, 0))])
    assert "no usable" in _create_error(m)


def test_too_many_bricks_is_unsupported():
    br = Brick([uniform_points(18), uniform_points(4), uniform_points(4)])
    m = split_brick(br, (list(range(2, 18, 2)), [], []))
    assert len(m.bricks) == 9
    assert "unsupported" in _create_error(m)


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_valid_multibrick_passes_the_host_checks():
    mesh, _, _ = workloads.multibrick(4)
    assert "no usable" in _create_error(mesh)


def test_dirichlet_and_gradients_on_multibrick_are_unsupported():
    bc = ("Dirichlet",) + ("Neumann",) * 5
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], bc, (0, 0, 0)),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], bc, (0, 8, 0))])
    assert "unsupported" in _create_error(m)
    vals = (0.0, 0.5, 0.0, 0.0, 0.0, 0.0)
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], ("Neumann",) * 6, (0, 0, 0), vals),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], ("Neumann",) * 6, (0, 8, 0))])
    assert "unsupported" in _create_error(m)


def test_unknown_face_type_and_bad_values_are_rejected():
    pts = [_pts(8, 0), _pts(8, 0), _pts(8, 0)]
    with pytest.raises(bb.FatalError, match="Incompatible boundary condition"):
        bb.Context(Mesh([Brick(pts, ("empty",) * 6)]), bb.make_options({}))
    bad = Brick(pts, ("Dirichlet",) + ("Neumann",) * 5, (0, 0, 0), (float("nan"),) + (0.0,) * 5)
    assert "invalid argument" in _create_error(Mesh([bad]))


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_single_brick_dirichlet_passes_the_host_checks():
    pts = [_pts(8, 0), _pts(8, 0), _pts(8, 0)]
    m = Mesh([Brick(pts, ("Dirichlet", "Neumann", "periodic", "periodic", "Neumann", "Dirichlet"),
                    (0, 0, 0), (1.0, 0.5, 0.0, 0.0, 0.0, -2.0))])
    assert "no usable" in _create_error(m)
