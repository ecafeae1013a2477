"""The flexible-CG outer loop (krylov fcg): FP64 residual and update, one
multigrid cycle (FP64 or FP32) as the preconditioner.  It must reach the
same solutions as the reference's cycle-by-cycle loop against independent
ground truths, in fewer cycles, with the reported residual recomputed from
the returned x."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from tests.helpers import channel_solution, dct_neumann_solution, rel, union_operator, union_solve, vmean

pytestmark = pytest.mark.gpu

KEYS = {"autotune": "off", "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2}


def _solve(mesh, b, **kw):
    d = dict(KEYS)
    d.update(kw)
    c = bb.Context(mesh, bb.make_options(d))
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    return x, rep


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fcg_cavity_matches_dct(native, precision):
    mesh, b, _ = workloads.cavity(32, seed=1000)
    br = mesh.bricks[0]
    x, rep = _solve(mesh, b, krylov="fcg", precision=precision, relTol=1e-12, coarseLevel=1)
    assert rep.status == 0
    xt = dct_neumann_solution(b.reshape(br.N), 1.0 / 32)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xt, V)) <= 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fcg_channel_fewer_cycles(native, precision):
    mesh, b, _ = workloads.channel(64, seed=2000)
    br = mesh.bricks[0]
    xr, rr = _solve(mesh, b, precision=precision, relTol=1e-10, coarseLevel=1)
    xk, rk = _solve(mesh, b, krylov="fcg", precision=precision, relTol=1e-10, coarseLevel=1)
    assert rr.status == 0 and rk.status == 0
    assert rk.cycles < 0.7 * rr.cycles
    xt = channel_solution(b.reshape(br.N), *br.points)
    V = br.cell_volumes()
    assert rel(vmean(xk.reshape(br.N), V), vmean(xt, V)) <= 1e-6
    assert rk.rel_residual <= 1.5e-10


def test_fcg_reported_residual_is_recomputed(native):
    mesh, b, _ = workloads.multibrick(4)
    A, V = union_operator(mesh)
    x, rep = _solve(mesh, b, krylov="fcg", precision="mixed", relTol=1e-8)
    assert rep.status == 0
    r = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert abs(r - rep.rel_residual) <= 1e-6 * r + 1e-15
    assert r <= 1.5e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fcg_multibrick_matches_union(native, precision):
    mesh, b, _ = workloads.multibrick(4)
    xref, V = union_solve(mesh, b)
    x, rep = _solve(mesh, b, krylov="fcg", precision=precision, relTol=1e-12, maxIter=100)
    assert rep.status == 0
    assert rel(x, xref) <= 1e-9


def test_fcg_variable_coefficient(native):
    mesh, b, lam = workloads.sphere(32, seed=4000)
    br = mesh.bricks[0]
    xs = {}
    for kr in ("none", "fcg"):
        c = bb.Context(mesh, bb.make_options(dict(KEYS, krylov=kr, relTol=1e-12, maxIter=300, coarseLevel=1)))
        c.set_coefficients(lam)
        x = np.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        assert rep.status == 0
        xs[kr] = (x, rep.cycles)
    assert xs["fcg"][1] < xs["none"][1]
    assert rel(xs["fcg"][0], xs["none"][0]) <= 1e-8


def test_fcg_graph_matches_host_loop(native):
    mesh, b, _ = workloads.channel(32, seed=7)
    out = {}
    for g in ("on", "off"):
        x, rep = _solve(mesh, b, krylov="fcg", precision="mixed", relTol=1e-9, coarseLevel=1, graph=g)
        assert rep.status == 0
        out[g] = (x, rep.cycles, rep.rel_residual)
    assert out["on"][1] == out["off"][1]
    assert np.array_equal(out["on"][0], out["off"][0]) and out["on"][2] == out["off"][2]


def test_fcg_repeat_is_deterministic(native):
    """Repeated solves give identical answers: no state leaks between solves
    (p and q start from whatever the last solve left)."""
    mesh, b, _ = workloads.channel(32, seed=8)
    c = bb.Context(mesh, bb.make_options(dict(KEYS, krylov="fcg", precision="mixed", relTol=1e-9,
                                              coarseLevel=1)))
    x1 = np.zeros_like(b)
    r1 = c.solve(b, x1, zero_guess=True)
    x2 = np.zeros_like(b)
    r2 = c.solve(b, x2, zero_guess=True)
    assert r1.cycles == r2.cycles and np.array_equal(x1, x2)
