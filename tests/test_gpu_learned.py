"""The learned initial guess: the ||b||-relative convergence test it relies
on, and what a trained network gains over the same solver started from
zero on held-out right-hand sides of the Taylor-Green sequence."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import learned, unet, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def built():
    from briscola_b200.build import build_unet

    build_unet()
    unet.load()


@pytest.mark.parametrize("krylov", ["none", "fcg"])
def test_rhs_criterion(native, krylov):
    mesh, b, _ = workloads.channel(32, seed=5)
    keys = {"relTol": 1e-8, "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2, "coarseLevel": 1,
            "krylov": krylov, "autotune": "off"}
    ci = bb.Context(mesh, bb.make_options(dict(keys, criterion="initial")))
    cr = bb.Context(mesh, bb.make_options(dict(keys, criterion="rhs")))
    x1, x2 = np.zeros_like(b), np.zeros_like(b)
    r1 = ci.solve(b, x1, zero_guess=True)
    r2 = cr.solve(b, x2, zero_guess=True)
    # from zero the two tests coincide
    assert r1.status == r2.status == 0 and r1.cycles == r2.cycles and np.array_equal(x1, x2)
    assert abs(r2.rhs_rel_residual - r2.rel_residual) <= 1e-12 and r2.rhs_rel_residual <= 1e-8
    # from a good guess the ||b|| test stops early, the reference's does not
    xg = x1 + 1e-6 * np.random.default_rng(0).standard_normal(b.size)
    ya, yb = xg.copy(), xg.copy()
    ra = ci.solve(b, ya)
    rb = cr.solve(b, yb)
    assert ra.status == rb.status == 0
    assert rb.cycles < ra.cycles and rb.rhs_rel_residual <= 1e-8


@pytest.fixture(scope="module")
def trained(built):
    """a network trained on 96 pairs of one 32^3 sequence"""
    N = 32
    train_set = learned.PairSet(N, 96, seed=1, every=2)
    net = unet.UNet((N,) * 3, seed=0)
    losses = learned.train(net, train_set, steps=2000, lr=2e-3)
    return net, train_set.scale, losses


def test_learned_guess_gain(native, trained):
    """Trained on 96 pairs of one sequence, judged on 8 pairs of another: the
    guess must be much closer to the solution than zero (the zero guess has
    relative error 1), leave no more residual than zero does, and never cost
    the solver a cycle.  At this size the preconditioned cycle removes ~20x
    of every error component per cycle, so the guess saves no whole cycle;
    the numbers are printed."""
    N = 32
    net, scale, losses = trained
    held = learned.PairSet(N, 8, seed=2, skip=40, every=5)
    assert np.mean(losses[-50:]) < 0.2 * np.mean(losses[:20]), (losses[:5], losses[-5:])
    ctx = bb.Context(learned.cube_mesh(N), bb.make_options(dict(learned.TARGET_KEYS, relTol=1e-8)))
    lg = learned.LearnedGuess(net, ctx, scale)
    n = N ** 3
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    cyc0, cyc1, err, res = [], [], [], []
    for q in range(len(held)):
        b = held.b[q]
        r0 = ctx.solve(b, x, zero_guess=True)
        xs = x.clone()
        r1 = lg.solve(b, x)
        assert r0.status == 0 and r1.status == 0
        assert r0.rhs_rel_residual <= 1e-8 and r1.rhs_rel_residual <= 1e-8
        cyc0.append(r0.cycles)
        cyc1.append(r1.cycles)
        # ||b - A x_guess|| / ||b||: the residual the cycles start from
        res.append(r1.rhs_rel_residual / r1.rel_residual)
        g = lg.x0 - lg.x0.mean()
        t = xs - xs.mean()
        err.append(float((g - t).norm() / t.norm()))
    print(f"cycles from zero {cyc0}, from the learned guess {cyc1}, guess error {np.round(err, 3)}, "
          f"guess residual {np.round(res, 3)}, final loss {np.mean(losses[-50:]):.3e}")
    assert np.mean(err) < 0.3
    assert np.mean(res) < 1.1
    assert all(c1 <= c0 for c0, c1 in zip(cyc0, cyc1))


def test_plugin_learned_guess_from_checkpoint(native, trained, tmp_path):
    """the GPUMG plugin with "learned guess;" loads the checkpoint and
    solves host arrays and device tensors to tolerance, on the training grid
    and on a finer one (the guess is scaled by (h / h_train)^2)"""
    net, scale, _ = trained
    path = str(tmp_path / "net.bunet")
    learned.save(net, scale, path, 32)
    for N in (32, 64):
        mesh = learned.cube_mesh(N)
        seq = workloads.TaylorGreenSequence(N, 7, torch.device("cuda", 0))
        b = seq.rhs()
        keys = dict(relTol=1e-8, tolerance=0, cycleType="V", nSweepsPre=2, nSweepsPost=2, coarseLevel=1,
                    precision="mixed", krylov="fcg")
        s_off = bb.solver.New(bb.Dictionary(dict(keys, type="GPUMG")), mesh)
        s_on = bb.solver.New(bb.Dictionary(dict(keys, type="GPUMG", learned="guess", learnedWeights=path)), mesh)
        x0 = torch.zeros_like(b)
        r0 = s_off.solve(bb.LinearSystem(mesh, x0, b, zero_guess=True))
        x1 = torch.zeros_like(b)
        r1 = s_on.solve(bb.LinearSystem(mesh, x1, b))
        bh = b.cpu().numpy()
        xh = np.zeros_like(bh)
        r2 = s_on.solve(bb.LinearSystem(mesh, xh, bh))
        for r in (r0, r1, r2):
            assert r.status == 0 and r.rhs_rel_residual <= 1e-8
        assert r1.cycles <= r0.cycles + 1 and r2.cycles == r1.cycles
        # the guess's own residual against ||b||: about that of zero on the
        # training grid; still of that order on the finer one (a guess
        # scaled wrongly by (h / h_train)^2 would leave several times ||b||)
        assert r1.rhs_rel_residual / r1.rel_residual < (1.5 if N == 32 else 3.0)
