"""coarseMode smooth (MG.C:110-126): the coarsest level of every cycle is
smoothed max(nSweepsPost, 2) times instead of solved directly, and on a
singular system the smoothers keep the pinned cell at zero, as the
reference's pinned coarse matrix does (solver.C:201-231, MG.C:37-40).
Against the oracle (oracle/bmg_oracle.cpp with coarse_direct = 0)."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import Brick, Mesh, geometric_points, uniform_points
from oracle.pyoracle import Oracle
from tests.helpers import rel, vmean

pytestmark = pytest.mark.gpu

V22 = dict(n_pre=2, n_post=2, cycle_type="V", coarse_direct=0)


def ctx(mesh, **kw):
    d = {"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseMode": "smooth"}
    d.update(kw)
    return bb.Context(mesh, bb.make_options(d))


@pytest.mark.parametrize("coarse_level", [1, 2])
def test_pinned_coarse_smoothing_matches_the_oracle(native, coarse_level):
    br = Brick([uniform_points(32), geometric_points(16, 2.0), uniform_points(16)])
    c = ctx(Mesh([br]), coarseLevel=coarse_level)
    o = Oracle(br.points, br.periodic, nthreads=4)
    o.assemble(coarse_level=coarse_level, **V22)
    lc = c.coarse_level_index
    rng = np.random.default_rng(1)
    x = rng.standard_normal(c.shape(lc))
    b = rng.standard_normal(c.shape(lc))
    x.flat[0] = 0.0  # the cycle zeroes x and the pinned b (MG.C:37-45)
    b.flat[0] = 0.0
    c.upload(lc, "x", x)
    c.upload(lc, "b", b)
    c.smooth(lc, 2)
    got = c.download(lc, "x")
    assert got.flat[0] == 0.0
    assert rel(got, o.smooth(lc, x, b, sweeps=2)) <= 1e-13


@pytest.mark.parametrize("wl", ["cavity", "channel"])
def test_solve_with_smoothed_coarse_level_matches_the_oracle(native, wl):
    mesh, b, _ = getattr(workloads, wl)(32)
    br = mesh.bricks[0]
    c = ctx(mesh, relTol=1e-12, maxIter=200, coarseLevel=1)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    xo, orep, _, rc = Oracle(br.points, br.periodic, nthreads=4).solve(
        b.reshape(br.N), rel_tol=1e-12, max_iter=200, stale_residual=0, coarse_level=1, **V22)
    assert rc == 0
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-9
    assert abs(rep.cycles - orep.iterations) <= 1, (rep.cycles, orep.iterations)


def test_fixed_cycles_with_a_large_smoothed_coarse_level(native):
    """A 16^3 coarse level smoothed twice is a poor coarse solver (the
    reference converges slowly there too); the same ten cycles give the
    oracle's iterate.  (All walls: on periodic axes the device's red-black
    order differs from the reference's padded sweep, so only the converged
    solutions agree there, as above.)"""
    mesh, b, _ = workloads.cavity(32)
    br = mesh.bricks[0]
    c = ctx(mesh, relTol=0.0, maxIter=10, coarseLevel=3)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.cycles == 10
    xo, orep, _, _ = Oracle(br.points, br.periodic, nthreads=4).solve(
        b.reshape(br.N), rel_tol=0.0, max_iter=10, stale_residual=0, coarse_level=3, **V22)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-11


def test_dirichlet_smoothed_coarse_level_and_large_coarse_levels(native):
    """No pin without singularity; and a coarse level above the dense
    solve's 4096 cells is fine when it is smoothed, refused when direct.
    (Dirichlet on every face: where a Dirichlet and a Neumann wall meet the
    device's prolongation differs from the reference's at the edge, so
    cycle-by-cycle iterates agree only without such edges.)"""
    vals = (1.0, -0.5, 0.25, 0.0, 2.0, -1.0)
    br = Brick([uniform_points(64)] * 3, ("Dirichlet",) * 6, values=vals)
    b = np.random.default_rng(2).standard_normal(int(np.prod(br.N)))
    c = ctx(Mesh([br]), relTol=0.0, maxIter=8, coarseLevel=4)  # coarse level 32^3
    assert int(np.prod(c.shape(c.coarse_level_index))) > 4096
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.cycles == 8
    xo, orep, _, _ = Oracle(br.points, br.periodic, nthreads=8, dirichlet=[True] * 6,
                            values=vals).solve(b.reshape(br.N), rel_tol=0.0, max_iter=8,
                                               stale_residual=0, coarse_level=4, **V22)
    # rounding only: the row-scaled device arithmetic against the oracle's
    # seven coefficients, over eight cycles that are far from converged
    assert rel(x, xo.ravel()) <= 1e-9
    with pytest.raises(bb.FatalError):
        ctx(Mesh([br]), coarseLevel=4, coarseMode="direct")


def test_mixed_fcg_with_smoothed_coarse_level(native):
    mesh, b, _ = workloads.channel(64)
    c = ctx(mesh, relTol=1e-8, precision="mixed", krylov="fcg", coarseLevel=2, maxIter=100)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0 and rep.rel_residual <= 1.5e-8


def test_refused_options_leave_the_context_unchanged(native):
    """bmg_set_options refuses a direct coarse solve on a level above 4096
    cells before it changes anything: the context keeps solving with the
    options it had."""
    mesh, b, _ = workloads.cavity(64)
    c = ctx(mesh, relTol=0.0, maxIter=5, coarseLevel=4)  # smoothed 32^3 coarse level
    with pytest.raises(bb.FatalError):
        c.set_options(bb.make_options({"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V",
                                       "coarseMode": "direct", "coarseLevel": 4}))
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.cycles == 5 and rep.final_residual < 0.5 * rep.initial_residual
