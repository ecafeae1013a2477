"""The projection steps either side of the pressure solve on the device
(bmg_project_rhs / bmg_project_correct in include/bmg.h) against their
restatement (oracle/fft_oracle.py: coloDiv, stagReconstruct), and whole
device-resident projection steps through the GPU multigrid and the GPU FFT
solver that leave a divergence-free velocity."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import fft
from briscola_b200.mesh import NEUMANN, PERIODIC, Brick, Mesh, geometric_points, uniform_points
from oracle import fft_oracle as F

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, P = NEUMANN, PERIODIC
BC = (P, P, N, N, P, P)
PER = (True, False, True)


def case(n=(16, 24, 16), seed=0):
    pts = [uniform_points(n[0]), geometric_points(n[1], 2.0), uniform_points(n[2])]
    rng = np.random.default_rng(seed)
    u = [rng.standard_normal((n[0] + 1, n[1], n[2])), rng.standard_normal((n[0], n[1] + 1, n[2])),
         rng.standard_normal((n[0], n[1], n[2] + 1))]
    u[0][-1] = u[0][0]
    u[2][:, :, -1] = u[2][:, :, 0]
    u[1][:, 0, :] = 0.0
    u[1][:, -1, :] = 0.0
    return pts, u, rng


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_rhs_and_correction_match_the_restatement():
    pts, u, rng = case()
    n = tuple(len(p) - 1 for p in pts)
    c = bb.Context(Mesh([Brick(pts, BC)]), bb.make_options({}))
    ud = [dev(a) for a in u]
    cdt = 0.05
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    c.project_rhs(ud, cdt, b, per_volume=True)
    ref = F.colo_div(u, pts) / (-cdt)
    assert rel(b.cpu().numpy(), ref) <= 1e-13
    c.project_rhs(ud, cdt, b)
    V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
    assert rel(b.cpu().numpy(), -V * ref) <= 1e-13
    p = rng.standard_normal(n)
    lam = [1.0 + rng.random(a.shape) for a in u]
    for lm in (None, lam):
        ud = [dev(a) for a in u]
        c.project_correct(ud, dev(p), cdt, None if lm is None else [dev(a) for a in lm])
        want = F.project_correct(u, p, cdt, pts, PER, lm)
        for d in range(3):
            assert rel(ud[d].cpu().numpy(), want[d]) <= 1e-13, d
    c.close()


@pytest.mark.parametrize("solver", ["GPUMG", "FFT"])
def test_device_resident_projection_is_divergence_free(solver):
    pts, u, _ = case((32, 48, 32), seed=1)
    n = tuple(len(p) - 1 for p in pts)
    mesh = Mesh([Brick(pts, BC)])
    c = bb.Context(mesh, bb.make_options({"relTol": 1e-13, "maxIter": 200, "coarseLevel": 1}))
    ud = [dev(a) for a in u]
    cdt = 0.05
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    p = torch.zeros_like(b)
    if solver == "GPUMG":
        c.project_rhs(ud, cdt, b)                 # system form for bmg_solve
        c.solve(b.view(-1), p.view(-1), zero_guess=True)
    else:
        c.project_rhs(ud, cdt, b, per_volume=True)  # the Poisson source for the FFT solver
        fft.FFTPoissonSolver(mesh.bricks[0]).solve(p, b)
    c.project_correct(ud, p, cdt)
    div = F.colo_div([a.cpu().numpy() for a in ud], pts)
    before = np.abs(F.colo_div(u, pts)).max()
    assert np.abs(div).max() <= (1e-9 if solver == "GPUMG" else 1e-11) * before
    c.close()
