"""GPU parity of the CUDA solver against the CPU oracle, through the C ABI.

Tolerances: FP64 kernels agree with the oracle to 1e-13 relative (the
device stores the operator row-scaled by 1/V, so the two differ by rounding
only); full FP64 solves agree to 1e-10 relative in the volume-weighted
mean-free solution (the bar for the plain FP64 path); FP32 kernels to 2e-6.
"""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import _native as NA
from briscola_b200 import workloads
from briscola_b200.mesh import NEUMANN, PERIODIC, Brick, Mesh, geometric_points, tanh_points, uniform_points
from oracle.pyoracle import Oracle
from tests.helpers import channel_solution, dct_neumann_solution, rel, vmean

pytestmark = pytest.mark.gpu

V22 = dict(n_pre=2, n_post=2, cycle_type="V", coarse_level=1)
DICT_V22 = {"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": 1}


def ctx_for(mesh, **kw):
    d = dict(DICT_V22)
    d.update(kw)
    return bb.Context(mesh, bb.make_options(d))


def oracle_for(br: Brick, lam=None):
    o = Oracle(br.points, periodic=br.periodic, nthreads=4)
    if lam is not None:
        o.set_lambda(*lam)
    return o


MESHES = {
    "uniform_walls": lambda: Brick([uniform_points(16), uniform_points(12), uniform_points(24)]),
    "graded_walls": lambda: Brick([geometric_points(16, 2.0), uniform_points(8), geometric_points(12, 0.5)]),
    "channel": lambda: Brick([uniform_points(16), tanh_points(16, 2.0), uniform_points(8)],
                             (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC)),
    "all_periodic": lambda: Brick([uniform_points(8), uniform_points(8), uniform_points(16)], (PERIODIC,) * 6),
}


def rand_lam(br, seed):
    rng = np.random.default_rng(seed)
    n0, n1, n2 = br.N
    return [np.exp(rng.uniform(-2, 2, s)) for s in ((n0 + 1, n1, n2), (n0, n1 + 1, n2), (n0, n1, n2 + 1))]


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("variable", [False, True])
def test_kernel_parity_fp64(native, name, variable):
    br = MESHES[name]()
    if variable and br.periodic[0]:
        lam = rand_lam(br, 1)
        for d in range(3):  # a periodic face is one face: both copies equal
            if br.periodic[d]:
                sl0 = [slice(None)] * 3
                sl1 = [slice(None)] * 3
                sl0[d], sl1[d] = 0, -1
                lam[d][tuple(sl1)] = lam[d][tuple(sl0)]
    else:
        lam = rand_lam(br, 1) if variable else None
    mesh = Mesh([br])
    c = ctx_for(mesh)
    if lam is not None:
        c.set_coefficients(lam)
    o = oracle_for(br, lam)
    lc = c.coarse_level_index
    o.assemble(**V22)
    rng = np.random.default_rng(7)
    for l in range(c.num_levels):
        shp = c.shape(l)
        assert shp == o.shape(l)
        x = rng.standard_normal(shp)
        b = rng.standard_normal(shp)
        if l == lc:
            continue
        # residual
        c.upload(l, "x", x)
        c.upload(l, "b", b)
        r_gpu = c.residual(l)
        r_ref = o.residual(l, x, b)
        assert rel(r_gpu, r_ref) <= 1e-13, ("residual", l)
        # colour passes
        for colour in (0, 1):
            c.upload(l, "x", x)
            c.colour_pass(l, colour)
            xg = c.download(l, "x")
            xr = o.colour_pass(l, colour, x, b)
            assert rel(xg, xr) <= 1e-13, ("colour", l, colour)
        if l + 1 < c.num_levels:
            # fused residual + restriction
            c.upload(l, "x", x)
            c.residual_restrict(l)
            bc_gpu = c.download(l + 1, "b")
            bc_ref = o.restrict(l, r_ref, scale=True)
            assert rel(bc_gpu, bc_ref) <= 1e-13, ("restrict", l)
            assert np.all(c.download(l + 1, "x") == 0.0)
            # fused prolongation + correction
            xc = rng.standard_normal(c.shape(l + 1))
            c.upload(l + 1, "x", xc)
            c.upload(l, "x", x)
            c.prolong_correct(l)
            xg = c.download(l, "x")
            xr = o.prolong(l, xc, x, op="+=")
            assert rel(xg, xr) <= 1e-13, ("prolong", l)


@pytest.mark.parametrize("name", ["uniform_walls", "channel"])
def test_coarse_solve_parity(native, name):
    br = MESHES[name]()
    c = ctx_for(Mesh([br]))
    o = oracle_for(br)
    o.assemble(**V22)
    lc = c.coarse_level_index
    rng = np.random.default_rng(3)
    b = rng.standard_normal(c.shape(lc))
    b.flat[0] = 0.0  # MG.C:37-40 pins b(0,0,0) on the coarse level
    c.upload(lc, "b", b)
    c.coarse_solve()
    xg = c.download(lc, "x")
    xr = o.coarse_solve(lc, b)
    assert rel(xg, xr) <= 1e-12


@pytest.mark.parametrize("name", list(MESHES))
def test_kernel_parity_fp32(native, name):
    br = MESHES[name]()
    c = ctx_for(Mesh([br]))
    o = oracle_for(br)
    o.assemble(**V22)
    rng = np.random.default_rng(11)
    # the coarse-solve level carries the singularity pin in the oracle's
    # matrix (solver.C:201-231); smoothers never run there
    for l in range(c.coarse_level_index):
        x = rng.standard_normal(c.shape(l))
        b = rng.standard_normal(c.shape(l))
        c.upload(l, "x", x, precision=1)
        c.upload(l, "b", b, precision=1)
        c.colour_pass(l, 0, precision=1)
        assert rel(c.download(l, "x", precision=1), o.colour_pass(l, 0, x, b)) <= 2e-6
        c.upload(l, "x", x, precision=1)
        c.residual_restrict(l, precision=1)
        assert rel(c.download(l + 1, "b", precision=1), o.restrict(l, o.residual(l, x, b))) <= 2e-6


def solve_gpu(mesh, b, lam=None, **kw):
    c = ctx_for(mesh, **kw)
    if lam is not None:
        c.set_coefficients(lam)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    return x, rep


@pytest.mark.parametrize("N", [32, 64])
def test_solve_cavity_matches_oracle(native, N):
    """Config 1 shape: all-wall cube, V(2,2), coarsest 4^3 direct."""
    mesh, b, _ = workloads.cavity(N, seed=1000)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, relTol=1e-13, maxIter=60)
    assert rep.status == 0
    xo, orep, _, rc = oracle_for(br).solve(b.reshape(br.N), rel_tol=1e-13, max_iter=60, **V22)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-10
    if N == 32:
        xt = dct_neumann_solution(b.reshape(br.N), 1.0 / N)
        assert rel(vmean(x.reshape(br.N), V), vmean(xt, V)) <= 1e-10


def test_solve_cavity_1e10_stop(native):
    """Config 1 stop criterion: 1e-10 relative residual; the GPU's cycle
    count matches the oracle without the stale-residual quirk (MG.C:72)."""
    mesh, b, _ = workloads.cavity(64, seed=1000)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, relTol=1e-10)
    assert rep.status == 0 and rep.final_residual / rep.initial_residual <= 1e-10
    xo, orep, hist, rc = oracle_for(br).solve(b.reshape(br.N), rel_tol=1e-10, stale_residual=0, **V22)
    assert abs(rep.cycles - orep.iterations) <= 1


@pytest.mark.parametrize("N", [32, 64])
def test_solve_channel_matches_oracle(native, N):
    mesh, b, _ = workloads.channel(N, seed=2000)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, relTol=1e-13, maxIter=80)
    assert rep.status == 0
    xo, orep, _, rc = oracle_for(br).solve(b.reshape(br.N), rel_tol=1e-13, max_iter=80, **V22)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-10
    xt = channel_solution(b.reshape(br.N), *br.points)
    assert rel(vmean(x.reshape(br.N), V), vmean(xt, V)) <= 1e-10


def test_solve_variable_coefficient_matches_oracle(native):
    mesh, b, lam = workloads.sphere(32, seed=4000)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, lam=lam, relTol=1e-13, maxIter=200)
    assert rep.status == 0
    o = oracle_for(br, lam)
    xo, orep, _, rc = o.solve(b.reshape(br.N), rel_tol=1e-13, max_iter=200, **V22)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-10


@pytest.mark.parametrize("cyc", ["W", "F"])
@pytest.mark.parametrize("smoother", ["rbgs", "jac"])
def test_cycles_and_smoothers(native, cyc, smoother):
    mesh, b, _ = workloads.channel(32, seed=5)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, relTol=1e-12, maxIter=200, cycleType=cyc, smoother=smoother)
    assert rep.status == 0
    xo, orep, _, rc = oracle_for(br).solve(b.reshape(br.N), rel_tol=1e-12, max_iter=200, n_pre=2,
                                           n_post=2, cycle_type=cyc, coarse_level=1, smoother=smoother)
    V = br.cell_volumes()
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-9


@pytest.mark.parametrize("wl", ["cavity", "channel"])
def test_mixed_precision_reaches_fp64_tolerance(native, wl):
    mesh, b, _ = workloads.CONFIGS[wl](64)
    br = mesh.bricks[0]
    x, rep = solve_gpu(mesh, b, relTol=1e-8, precision="mixed")
    assert rep.status == 0
    assert rep.rel_residual <= 1e-8
    x64, rep64 = solve_gpu(mesh, b, relTol=1e-13, maxIter=80)
    V = br.cell_volumes()
    err = rel(vmean(x.reshape(br.N), V), vmean(x64.reshape(br.N), V))
    assert err <= 1e-6, err


def test_reference_plugin_path(native):
    """solver.New(dict) -> GPUMG.solve(sys) as a Briscola case would call it."""
    mesh, b, _ = workloads.cavity(32, seed=2)
    d = bb.Dictionary.parse("""
        type GPUMG; relTol 1e-10; tolerance 0; cycleType V;
        nSweepsPre 2; nSweepsPost 2; coarseLevel 1; coarseMode direct;
        coarseSolver { type APLU; } smoother rbgs; restrict linear; prolong linear;""")
    s = bb.solver.New(d, mesh)
    x = np.zeros_like(b)
    rep = s.solve(bb.LinearSystem(mesh, x, b))
    assert rep.status == 0 and np.any(x != 0)
    assert rep.final_residual / rep.initial_residual <= 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_solve_on_legacy_default_stream(native, precision):
    """The whole-solve graph is captured on a private stream and launched
    on the caller's, which may be the legacy default stream (torch's)."""
    mesh, b, _ = workloads.channel(32, seed=6)
    c = ctx_for(mesh, relTol=1e-8, precision=precision)
    c.set_stream(0)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0 and rep.rel_residual <= 1e-8
    c2 = ctx_for(mesh, relTol=1e-8, precision=precision, graph="off")
    x2 = np.zeros_like(b)
    rep2 = c2.solve(b, x2, zero_guess=True)
    assert rep2.cycles == rep.cycles and np.array_equal(x, x2)


def test_status_codes(native):
    mesh, b, _ = workloads.cavity(16, seed=3)
    # not converged within maxIter
    x, rep = solve_gpu(mesh, b, relTol=1e-14, maxIter=2)
    assert rep.status == NA.NOT_CONVERGED and rep.cycles == 2
    # NaN in the right-hand side
    bn = b.copy()
    bn[5] = np.nan
    x, rep = solve_gpu(mesh, bn, relTol=1e-8)
    assert rep.status == NA.NAN_DETECTED
    # zero right-hand side: converged at once (solver.C:78 init = 0)
    x, rep = solve_gpu(mesh, np.zeros_like(b), relTol=1e-8)
    assert rep.status == 0 and rep.cycles == 0 and np.all(x == 0)
    # a time budget that cannot be met ends the loop with TIMEOUT
    x, rep = solve_gpu(mesh, b, relTol=1e-14, maxIter=100000, timeoutMs=1e-3)
    assert rep.status == NA.TIMEOUT


def test_initial_guess_is_used(native):
    """A warm start is judged like the reference judges it: the relative
    criterion is relative to the initial residual (solver.C:64-95), so a
    converged guess only stops at once through the absolute tolerance."""
    mesh, b, _ = workloads.cavity(32, seed=4)
    c = ctx_for(mesh, relTol=1e-12, tolerance=1e-11)
    x = np.zeros_like(b)
    rep0 = c.solve(b, x, zero_guess=True)
    rep1 = c.solve(b, x)
    assert rep0.cycles > 3 and rep0.status == 0
    assert rep1.cycles == 0 and rep1.status == 0
    # relative criterion only: a converged guess cannot improve by relTol
    c2 = ctx_for(mesh, relTol=1e-8, maxIter=5)
    rep2 = c2.solve(b, x)
    assert rep2.status == NA.NOT_CONVERGED and rep2.cycles == 5


def test_semicoarsening_shapes(native):
    """Extents of 2 and 3 stop coarsening in one direction (utils.H:1152-1170)."""
    br = Brick([uniform_points(32), uniform_points(6), uniform_points(3)])
    mesh = Mesh([br])
    rng = np.random.default_rng(1)
    V = br.cell_volumes()
    f = rng.standard_normal(br.N)
    f -= (V * f).sum() / V.sum()
    b = (-V * f).ravel()
    x, rep = solve_gpu(mesh, b, relTol=1e-12, maxIter=400, coarseLevel=0)
    assert rep.status == 0
    xo, orep, _, rc = oracle_for(br).solve(b.reshape(br.N), rel_tol=1e-12, max_iter=400, n_pre=2,
                                           n_post=2, cycle_type="V", coarse_level=0)
    assert rel(vmean(x.reshape(br.N), V), vmean(xo, V)) <= 1e-9


def test_device_solve_waits_for_the_producer_of_b(native):
    """b produced by torch work still queued on the current stream: the
    solve must run behind it (Context.solve follows torch's current stream)."""
    import torch

    mesh, b_np, _ = workloads.cavity(64, seed=3)
    b0 = torch.from_numpy(b_np).cuda()
    c = ctx_for(mesh, relTol=1e-10, criterion="rhs", krylov="fcg")
    for q in range(3):
        torch.cuda._sleep(50_000_000)  # keep the stream busy for tens of ms
        b = b0 * float(q + 1)          # written only after the sleep
        x = torch.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        assert rep.status == 0 and rep.rhs_rel_residual <= 1e-10
