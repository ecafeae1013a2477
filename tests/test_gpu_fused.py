"""The fused smoother (all colour passes of a smoothing step in one launch)
against the same passes launched one by one.  Both use the same stencil
arithmetic (bmg_stencil.cuh), so the results must be bit-identical, in FP64
and FP32, with constant and variable coefficients, walls and periodic axes,
and for sequences longer than one fused launch.  The fused smoother works on
natural rows, so these contexts keep rowLayout natural (parity-split levels
take the per-colour split kernel instead, tests/test_gpu_layout.py)."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import NEUMANN, PERIODIC, Brick, Mesh, geometric_points, tanh_points, uniform_points

pytestmark = pytest.mark.gpu

BRICKS = {
    "channel": lambda: Brick([uniform_points(64), tanh_points(48, 2.0), uniform_points(64)],
                             (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC)),
    "walls_graded": lambda: Brick([geometric_points(48, 2.0), uniform_points(48), geometric_points(96, 0.5)]),
    "all_periodic": lambda: Brick([uniform_points(32), uniform_points(32), uniform_points(32)], (PERIODIC,) * 6),
    # partial tiles in every direction: 96 planes = 64 + 32, 24 rows = 16 + 8, 48 columns < 64
    "odd_tiles": lambda: Brick([uniform_points(96), uniform_points(24), uniform_points(48)]),
}


def _lam(br, seed):
    rng = np.random.default_rng(seed)
    n0, n1, n2 = br.N
    lam = [np.exp(rng.uniform(-3, 3, s)) for s in ((n0 + 1, n1, n2), (n0, n1 + 1, n2), (n0, n1, n2 + 1))]
    for d in range(3):
        if br.periodic[d]:
            a = [slice(None)] * 3
            z = [slice(None)] * 3
            a[d], z[d] = -1, 0
            lam[d][tuple(a)] = lam[d][tuple(z)]
    return lam


@pytest.mark.parametrize("name", list(BRICKS))
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("variable", [False, True])
@pytest.mark.parametrize("stages", [1, 2, 3])
def test_fused_smoothing_bit_identical(native, name, precision, variable, stages):
    br = BRICKS[name]()
    mesh = Mesh([br])
    ctx = {f: bb.Context(mesh, bb.make_options({"fused": f, "autotune": "off", "coarseLevel": 1, "rowLayout": "natural"}))
           for f in (str(stages), "off")}
    ctx["on"] = ctx.pop(str(stages))
    assert ctx["on"].tuning(0, precision)[0] == stages and ctx["off"].tuning(0, precision)[0] == 0
    if variable:
        lam = _lam(br, 3)
        for c in ctx.values():
            c.set_coefficients(lam)
    rng = np.random.default_rng(5)
    for l in range(ctx["on"].num_levels):
        shp = ctx["on"].shape(l)
        if min(shp) < 16:
            break
        x = rng.standard_normal(shp)
        b = rng.standard_normal(shp)
        for sweeps in (1, 2, 3):  # 3, 5 and 7 colour stages (7 = two fused launches)
            out = {}
            for f, c in ctx.items():
                c.upload(l, "x", x, precision)
                c.upload(l, "b", b, precision)
                c.smooth(l, sweeps, precision)
                out[f] = c.download(l, "x", precision)
            assert np.array_equal(out["on"], out["off"]), (l, sweeps)
            # and the ghost images are consistent: a residual reads them
            res = {f: c.residual(l, precision) for f, c in ctx.items()}
            assert np.array_equal(res["on"], res["off"]), (l, sweeps)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_solve_bit_identical(native, precision):
    mesh, b, _ = workloads.channel(64, seed=8)
    xs, reps = {}, {}
    for f in ("on", "off"):
        c = bb.Context(mesh, bb.make_options({"fused": f, "autotune": "off", "relTol": 1e-10, "rowLayout": "natural",
                                              "nSweepsPre": 2, "nSweepsPost": 2,
                                              "cycleType": "V", "coarseLevel": 1, "precision": precision}))
        x = np.zeros_like(b)
        reps[f] = c.solve(b, x, zero_guess=True)
        xs[f] = x
    assert reps["on"].status == 0 and reps["on"].cycles == reps["off"].cycles
    assert np.array_equal(xs["on"], xs["off"])
    assert reps["on"].kernel_launches < reps["off"].kernel_launches


def test_autotuner_picks_valid_shapes(native):
    mesh, b, _ = workloads.channel(64, seed=9)
    c = bb.Context(mesh, bb.make_options({"nSweepsPre": 2, "nSweepsPost": 2, "coarseLevel": 1,
                                          "rowLayout": "natural"}))
    for l in range(c.num_levels):
        for p in (0, 1):
            s, t = c.tuning(l, p)
            if min(c.shape(l)) >= 16 and s > 0:
                assert s <= 3 and (t in (16, 24, 32, 48, 64, 128) or t == c.shape(l)[0])
            else:
                assert (s, t) == (0, 0)  # smoothed pass by pass
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    assert rep.status == 0


def test_pinned_launch_shapes(native):
    mesh, b, _ = workloads.channel(64, seed=10)
    c = bb.Context(mesh, bb.make_options({"coarseLevel": 1, "autotune": "off", "precision": "mixed",
                                          "rowLayout": "natural"}))
    c.set_tuning(0, 1, 2, 24)
    c.set_tuning(0, 0, 0, 64)
    assert c.tuning(0, 1) == (2, 24) and c.tuning(0, 0) == (0, 0)
    with pytest.raises(bb.FatalError):
        c.set_tuning(0, 1, 4, 24)  # more stages than a launch runs
    with pytest.raises(bb.FatalError):
        c.set_tuning(0, 1, 3, 0)  # chunk outside 1..128
    coarsest = c.num_levels - 1
    with pytest.raises(bb.FatalError):
        c.set_tuning(coarsest, 1, 3, 16)  # a level the fused smoother does not handle
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    ref = bb.Context(mesh, bb.make_options({"coarseLevel": 1, "fused": "off", "precision": "mixed",
                                            "rowLayout": "natural"}))
    x2 = np.zeros_like(b)
    rep2 = ref.solve(b, x2, zero_guess=True)
    assert rep.status == 0 and rep.cycles == rep2.cycles and np.array_equal(x, x2)
