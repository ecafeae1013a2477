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


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_dirichlet_and_gradients_on_multibrick_walls_pass_the_host_checks():
    bc = ("Dirichlet",) + ("Neumann",) * 5
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], bc, (0, 0, 0)),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], bc, (0, 8, 0))])
    assert "no usable" in _create_error(m)
    vals = (0.0, 0.5, 0.0, 0.0, 0.0, 0.0)
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], ("Neumann",) * 6, (0, 0, 0), vals),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], ("Neumann",) * 6, (0, 8, 0))])
    assert "no usable" in _create_error(m)
    # faces wholly in contact are interfaces: their own conditions are ignored
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], ("Dirichlet",) * 6, (0, 0, 0), (1.0,) * 6),
              Brick([_pts(8, 0), _pts(8, 8), _pts(8, 0)], ("Dirichlet",) * 6, (0, 8, 0), (2.0,) * 6)])
    assert "no usable" in _create_error(m)


def test_conditions_on_faces_partly_in_contact_are_unsupported():
    """brick 0's upper y face touches brick 1 over half its width; the other
    half is a zero-gradient wall, which cannot take a Dirichlet value or a
    gradient (the reference links whole faces only)"""
    lower, upper = (0, 0, 0), (0, 8, 0)
    for bc, vals in ((("Neumann",) * 3 + ("Dirichlet",) + ("Neumann",) * 2, (0.0,) * 6),
                     (("Neumann",) * 6, (0.0, 0.0, 0.0, 0.25, 0.0, 0.0))):
        m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], bc, lower, vals),
                  Brick([_pts(4, 0), _pts(8, 8), _pts(8, 0)], ("Neumann",) * 6, upper)])
        assert "unsupported" in _create_error(m)


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_partial_contact_with_zero_gradient_walls_passes_the_host_checks():
    m = Mesh([Brick([_pts(8, 0), _pts(8, 0), _pts(8, 0)], ("Neumann",) * 6, (0, 0, 0)),
              Brick([_pts(4, 0), _pts(8, 8), _pts(8, 0)], ("Dirichlet",) + ("Neumann",) * 5, (0, 8, 0), (1.0,) * 6)])
    assert "no usable" in _create_error(m)


def test_union_operator_with_walls_of_split_brick_is_the_brick_operator():
    from tests.helpers import brick_operator, union_operator_bc

    pts = [uniform_points(8), geometric_points(6, 2.0), uniform_points(4)]
    bc = ("Dirichlet", "Neumann", "Neumann", "Dirichlet", "Neumann", "Neumann")
    vals = (1.0, 0.5, -0.25, 2.0, 0.0, 0.75)
    br = Brick(pts, bc, values=vals)
    A0, V0, b0 = brick_operator(pts, bc, vals)
    A1, V1, b1 = union_operator_bc(Mesh([br]))
    assert abs(A1 - A0).max() < 1e-15 and np.abs(b1 - b0).max() < 1e-15
    parts = split_brick(br, ([4], [3], [2]))
    A2, V2, b2 = union_operator_bc(parts)
    perm = brick_to_compact(parts, np.arange(8 * 6 * 4).reshape(8, 6, 4))
    assert abs(A0[perm][:, perm] - A2).max() < 1e-15 and np.abs(b0[perm] - b2).max() < 1e-15


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
