"""Learned initial guess for the multigrid solve.

Training pairs come from the plain GPU multigrid itself: a time sequence of
right-hand sides (``workloads.TaylorGreenSequence``) is solved to a tight
tolerance and each (b, x) pair is stored normalised -- input -b / rms(b),
target x V / rms(b), divided by one RMS for the whole set -- so that the network maps a unit-size source to its
solution; the solution is linear in b, so the guess for any b is the network
output scaled back.  The U-Net (``unet.UNet``) trains on its own kernels.

``LearnedGuess.solve`` runs the network, then the solver from that guess
with the convergence test relative to ||b|| (``criterion rhs``), so the
guess can only help by leaving less residual for the cycles to remove; the
solver always finishes to tolerance.
"""
from __future__ import annotations

import math

import numpy as np

from . import unet as U
from . import workloads
from .mesh import Brick, Mesh, uniform_points
from .solvers import Context, make_options

# solver used to generate the training targets
TARGET_KEYS = {"relTol": 1e-10, "tolerance": 0, "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2,
               "coarseLevel": 1, "precision": "mixed", "krylov": "fcg", "criterion": "rhs"}


def cube_mesh(N: int) -> Mesh:
    return Mesh([Brick([uniform_points(N)] * 3)])


class PairSet:
    """Normalised (input, target) pairs on the device, FP32."""

    def __init__(self, N: int, count: int, seed: int, device=None, skip: int = 0, every: int = 1):
        import torch

        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.N = N
        self.V = (1.0 / N) ** 3
        mesh = cube_mesh(N)
        ctx = Context(mesh, make_options(dict(TARGET_KEYS, device=dev.index or 0)))
        seq = workloads.TaylorGreenSequence(N, seed, dev)
        for _ in range(skip):
            seq.step()
        n = N ** 3
        self.inputs = torch.zeros(count, n, dtype=torch.float32, device=dev)
        self.targets = torch.zeros(count, n, dtype=torch.float32, device=dev)
        self.b = []
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        self.cycles = []
        for q in range(count):
            b = seq.rhs()
            rep = ctx.solve(b, x, zero_guess=True)
            if rep.status != 0:
                raise RuntimeError(f"target solve failed: status {rep.status}")
            self.cycles.append(rep.cycles)
            rms = float(torch.sqrt(torch.mean(b * b)))
            self.inputs[q] = (-b / rms).float()
            self.targets[q] = (x * (self.V / rms)).float()
            self.b.append(b.clone())
            for _ in range(every):
                seq.step()
        ctx.close()
        # targets at unit RMS over the set; the guess multiplies back
        self.scale = float(torch.sqrt(torch.mean(self.targets.double() ** 2)))
        self.targets /= self.scale

    def __len__(self):
        return self.inputs.shape[0]


def train(net: U.UNet, pairs: PairSet, steps: int, lr: float = 1e-3, seed: int = 0, lr_final: float = 1e-4,
          res_weight: float = 1.0):
    """Adam on single pairs in a seeded random order; cosine learning rate
    from lr to lr_final.  The loss is the MSE of the normalised solution plus
    res_weight times the mean squared h^2-scaled operator residual of the
    output (A'y = -input / scale on the normalised pair), which penalises
    the rough errors that the MSE tolerates but that dominate the residual
    the solver starts from.  Returns the MSE of every step (host floats)."""
    h2 = (1.0 / pairs.N) ** 2
    res_c = h2 / pairs.scale
    rng = np.random.default_rng(seed)
    losses = []
    order = []
    for s in range(steps):
        if not order:
            order = list(rng.permutation(len(pairs)))
        q = order.pop()
        a = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * s / max(1, steps)))
        losses.append(net.train_step(pairs.inputs[q], pairs.targets[q], lr=a, res_c=res_c,
                                     res_weight=res_weight).clone())
    net.check_errors()
    return [float(v.item()) for v in losses]


def save(net: U.UNet, pairs_scale: float, path: str, N: int) -> None:
    """checkpoint with what LearnedGuess needs: the target scale and grid"""
    net.save(path, meta={"target_scale": pairs_scale, "training_grid": N})


class LearnedGuess:
    """A trained network in front of a solver context on the same N^3 cube."""

    def __init__(self, net: U.UNet, ctx: Context, scale: float, h: float | None = None, h_train: float | None = None):
        """scale: the target scale of the training pairs; h: the cell size of
        the grids solved (default 1/N, the unit cube); h_train: the cell
        size trained on (default h).  The network learned the solution of
        unit-size sources on the training grid; the solution grows with h^2,
        hence the factor (h / h_train)^2."""
        import torch

        self.torch = torch
        self.net = net
        self.ctx = ctx
        self.N = net.shape[0]
        h = 1.0 / self.N if h is None else h
        h_train = h if h_train is None else h_train
        self.V = h ** 3
        self.scale = scale * (h / h_train) ** 2
        self.x0 = torch.zeros(self.N ** 3, dtype=torch.float64, device=net.dev)

    def guess(self, b):
        return self.net.guess(b, self.V, self.x0, self.scale)

    def solve(self, b, x):
        """x = guess(b), then the solver from x; returns the solver report"""
        self.guess(b)
        x.copy_(self.x0)
        return self.ctx.solve(b, x, zero_guess=False)


def benchmark(N: int, n_pairs: int, steps: int, n_held: int, seed: int = 1, lr: float = 1e-3):
    """Config 5 as one measurement: train on n_pairs solved pairs of one
    sequence, then time held-out solves of another sequence from zero and
    from the learned guess (mixed precision, flexible CG, ||b||-relative
    1e-8).  Returns a dict of the timings and cycle counts (CUDA events)."""
    import time

    import torch

    t0 = time.perf_counter()
    pairs = PairSet(N, n_pairs, seed=seed)
    t_data = time.perf_counter() - t0
    net = U.UNet((N,) * 3, seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = train(net, pairs, steps, lr=lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    scale = pairs.scale
    del pairs
    torch.cuda.empty_cache()
    held = PairSet(N, n_held, seed=seed + 1000, skip=17, every=3)
    ctx = Context(cube_mesh(N), make_options(dict(TARGET_KEYS, relTol=1e-8)))
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    lg = LearnedGuess(net, ctx, scale)
    x = torch.zeros(N ** 3, dtype=torch.float64, device=net.dev)
    for q in range(min(3, n_held)):  # warm-up (graph capture, guess buffers)
        ctx.solve(held.b[q], x, zero_guess=True)
        lg.solve(held.b[q], x)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    cyc0, cyc1 = [], []
    torch.cuda.synchronize()
    e[0].record(stream)
    for q in range(n_held):
        cyc0.append(ctx.solve(held.b[q], x, zero_guess=True).cycles)
    e[1].record(stream)
    for q in range(n_held):
        cyc1.append(lg.solve(held.b[q], x).cycles)
    e[2].record(stream)
    for q in range(n_held):
        lg.guess(held.b[q])
    e[3].record(stream)
    torch.cuda.synchronize()
    net.check_errors()
    return {"grid": [N] * 3, "training_pairs": n_pairs, "training_steps": steps, "held_out": n_held,
            "data_s": round(t_data, 1), "train_s": round(t_train, 1),
            "final_loss": float(np.mean(losses[-50:])),
            "zero_guess": {"ms_per_solve": round(e[0].elapsed_time(e[1]) / n_held, 3),
                           "cycles_mean": float(np.mean(cyc0))},
            "learned_guess": {"ms_per_solve": round(e[1].elapsed_time(e[2]) / n_held, 3),
                              "cycles_mean": float(np.mean(cyc1)),
                              "guess_ms": round(e[2].elapsed_time(e[3]) / n_held, 3)}}
