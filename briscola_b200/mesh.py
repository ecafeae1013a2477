"""Rectilinear brick meshes: vertex coordinates per axis and face boundary
conditions, the part of a Briscola ``briscolaMeshDict`` the solver needs.

Gradings follow the reference where it has them:
``geometric`` -- src/briscolaMesh/gradings/geometricGrading/geometricGrading.C:43-71,
``none`` -- uniform.  The reference has no tanh grading; ``tanh_points``
gives the wall-clustered channel distribution y_j = (1 + tanh(g(2j/N - 1))/tanh g)/2.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NEUMANN = "Neumann"
PERIODIC = "periodic"
# Dirichlet faces: both solvers (on a multi-brick mesh, the multigrid takes
# them on brick faces that touch no other brick);
# empty axes: the FFT Poisson solver only (briscola_b200.fft)
DIRICHLET = "Dirichlet"
EMPTY = "empty"


def uniform_points(n: int, length: float = 1.0, start: float = 0.0) -> np.ndarray:
    return start + length * np.arange(n + 1, dtype=np.float64) / n


def geometric_points(n: int, ratio: float, length: float = 1.0, start: float = 0.0) -> np.ndarray:
    """geometricGrading.C:43-71: last-to-first cell size ratio ``ratio``."""
    f = np.arange(n + 1, dtype=np.float64) / n
    if n == 1:
        return start + length * f
    g = ratio ** (1.0 / (n - 1.0))
    if g == 1.0:
        return start + length * f
    d = (g - 1.0) / (g * (g ** (n - 1) - 1.0))
    return start + length * (d * g * (g ** (f * (n - 1)) - 1.0) / (g - 1.0))


def tanh_points(n: int, gamma: float, length: float = 1.0, start: float = 0.0) -> np.ndarray:
    """Wall-clustered points on [start, start+length] with stretching gamma."""
    j = np.arange(n + 1, dtype=np.float64)
    y = 0.5 * (1.0 + np.tanh(gamma * (2.0 * j / n - 1.0)) / np.tanh(gamma))
    y[0], y[-1] = 0.0, 1.0
    return start + length * y


@dataclass
class Brick:
    """One brick: ``points`` holds the vertex coordinates per axis; ``bc`` the
    boundary type of faces x-lo, x-hi, y-lo, y-hi, z-lo, z-hi; ``values`` the
    (uniform) Dirichlet value or Neumann gradient of each face; ``transform``
    the orientation of the brick's own frame in the mesh (local axis d runs
    along mesh axis |t_d| - 1, reversed when t_d < 0; zeros: the mesh's
    frame).  Points, faces, values and the brick's arrays are in its own
    frame, ``origin`` in the mesh's."""

    points: list
    bc: tuple = (NEUMANN,) * 6
    origin: tuple = (0, 0, 0)
    values: tuple = (0.0,) * 6
    transform: tuple = (0, 0, 0)

    def __post_init__(self):
        self.points = [np.ascontiguousarray(p, dtype=np.float64) for p in self.points]
        if len(self.points) != 3 or len(self.bc) != 6 or len(self.values) != 6:
            raise ValueError("a brick needs three coordinate arrays, six face conditions and six face values")

    @property
    def N(self):
        return tuple(len(p) - 1 for p in self.points)

    @property
    def periodic(self):
        return tuple(self.bc[2 * d] == PERIODIC for d in range(3))

    def cell_sizes(self, axis: int) -> np.ndarray:
        return np.abs(np.diff(self.points[axis]))  # points decrease along a reversed axis

    def cell_centres(self, axis: int) -> np.ndarray:
        p = self.points[axis]
        return 0.5 * (p[1:] + p[:-1])

    def cell_volumes(self) -> np.ndarray:
        hx, hy, hz = (self.cell_sizes(d) for d in range(3))
        return hx[:, None, None] * hy[None, :, None] * hz[None, None, :]


@dataclass
class Mesh:
    bricks: list = field(default_factory=list)

    @property
    def n_cells(self) -> int:
        return int(sum(np.prod(b.N) for b in self.bricks))


def box(N, lengths=(1.0, 1.0, 1.0), bc=(NEUMANN,) * 6, points=None) -> Mesh:
    """Single-brick mesh with uniform spacing unless ``points`` is given."""
    if points is None:
        points = [uniform_points(N[d], lengths[d]) for d in range(3)]
    return Mesh([Brick(points, tuple(bc))])
