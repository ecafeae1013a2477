"""B200-native geometric-multigrid Poisson solver for Briscola brick meshes.

``solver.New(dict, mesh)`` with ``type GPUMG;`` selects it, as a case's
``briscolaSolverDict`` selects the reference's ``MG``.  The solve runs in
hand-written sm_100a kernels behind the C ABI of ``include/bmg.h``.
"""
from .mesh import Brick, Mesh, box, geometric_points, tanh_points, uniform_points  # noqa: F401
from .solvers import GPUMG, Context, Dictionary, FatalError, LinearSystem, make_options, solver  # noqa: F401

__all__ = [
    "Brick", "Mesh", "box", "geometric_points", "tanh_points", "uniform_points",
    "GPUMG", "Context", "Dictionary", "FatalError", "LinearSystem", "make_options", "solver",
]
