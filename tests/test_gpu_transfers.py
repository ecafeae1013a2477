"""The other grid transfers of the reference's MG (MG.C:289-305): restrict
average (averageRestrictionScheme.C:17-77) and prolong injection
(injectionProlongationScheme.C:14-33), per kernel and in whole solves,
against the oracle."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import NEUMANN, PERIODIC, Brick, Mesh, geometric_points, uniform_points
from oracle.pyoracle import Oracle
from tests.helpers import rel, vmean

pytestmark = pytest.mark.gpu

SCHEMES = [("average", "linear"), ("linear", "injection"), ("average", "injection")]


def _ctx(mesh, restrict, prolong, **kw):
    d = {"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": 1, "restrict": restrict,
         "prolong": prolong}
    d.update(kw)
    return bb.Context(mesh, bb.make_options(d))


def _okw(restrict, prolong):
    return dict(restrict_average=int(restrict == "average"), prolong_injection=int(prolong == "injection"))


@pytest.mark.parametrize("restrict,prolong", SCHEMES)
def test_transfer_kernels_match_the_oracle(native, restrict, prolong):
    br = Brick([uniform_points(32), geometric_points(16, 2.0), geometric_points(24, 0.5)],
               (PERIODIC, PERIODIC, NEUMANN, NEUMANN, NEUMANN, NEUMANN))
    c = _ctx(Mesh([br]), restrict, prolong)
    o = Oracle(br.points, br.periodic, nthreads=4)
    o.assemble(n_pre=2, n_post=2, cycle_type="V", coarse_level=1, **_okw(restrict, prolong))
    rng = np.random.default_rng(3)
    for l in range(c.coarse_level_index):
        x = rng.standard_normal(c.shape(l))
        b = rng.standard_normal(c.shape(l))
        c.upload(l, "x", x)
        c.upload(l, "b", b)
        c.residual_restrict(l)
        assert rel(c.download(l + 1, "b"), o.restrict(l, o.residual(l, x, b), scale=True)) <= 1e-13, l
        xc = rng.standard_normal(c.shape(l + 1))
        c.upload(l + 1, "x", xc)
        c.upload(l, "x", x)
        c.prolong_correct(l)
        assert rel(c.download(l, "x"), o.prolong(l, xc, x, op="+=")) <= 1e-13, l


@pytest.mark.parametrize("restrict,prolong", SCHEMES)
@pytest.mark.parametrize("wl", ["cavity", "channel"])
def test_solves_match_the_oracle(native, restrict, prolong, wl):
    mesh, b, _ = getattr(workloads, wl)(32)
    br = mesh.bricks[0]
    c = _ctx(mesh, restrict, prolong, relTol=1e-12, maxIter=300)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0
    xo, orep, _, rc = Oracle(br.points, br.periodic, nthreads=4).solve(
        b.reshape(br.N), rel_tol=1e-12, max_iter=300, stale_residual=0, n_pre=2, n_post=2, cycle_type="V",
        coarse_level=1, **_okw(restrict, prolong))
    assert rc == 0
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-9
    if wl == "cavity":
        assert abs(rep.cycles - orep.iterations) <= 1, (rep.cycles, orep.iterations)
    else:
        # on periodic axes the device's red-black order differs from the
        # reference's padded sweep; with injection (a weak prolongation, ~60
        # cycles to 1e-12) that shows in the cycle count
        assert abs(rep.cycles - orep.iterations) <= 0.2 * orep.iterations, (rep.cycles, orep.iterations)


def test_switching_schemes_rebuilds_the_tables(native):
    mesh, b, _ = workloads.channel(32)
    fresh = _ctx(mesh, "average", "injection", relTol=1e-10)
    x1 = np.zeros_like(b)
    r1 = fresh.solve(b, x1, zero_guess=True)
    c = _ctx(mesh, "linear", "linear", relTol=1e-10)
    c.solve(b, np.zeros_like(b), zero_guess=True)
    c.set_options(bb.make_options({"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": 1,
                                   "restrict": "average", "prolong": "injection", "relTol": 1e-10}))
    x2 = np.zeros_like(b)
    r2 = c.solve(b, x2, zero_guess=True)
    assert r1.cycles == r2.cycles
    assert np.array_equal(x1, x2)


def test_mixed_fcg_with_the_other_transfers(native):
    mesh, b, _ = workloads.channel(64)
    c = _ctx(mesh, "average", "injection", relTol=1e-8, precision="mixed", krylov="fcg", maxIter=100)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0 and rep.rel_residual <= 1.5e-8
