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

``CoarseCorrection`` puts a network trained on one level of the hierarchy
in place of the multigrid recursion below that level (the restricted
residual in, the level's correction out, then the level's post-smoothing;
MG.C:77-99 is the recursion it replaces) in the FP32 cycles of a
mixed-precision solve.  Its training pairs are the right-hand sides that
level actually receives during solves of the sequence, with the level's
exact solutions as targets (``CoarsePairSet``).  The outer FP64 loop still
decides convergence, so the solve always finishes to tolerance.
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


class _DeviceArray:
    """A raw device pointer as an object torch can view without a copy."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, n: int, dtype=None):
    """A torch CUDA tensor aliasing n elements at the device pointer ptr
    (FP32 unless dtype says otherwise)."""
    import torch

    dtype = dtype or torch.float32
    typestr = {torch.float32: "<f4", torch.float64: "<f8"}[dtype]
    return torch.as_tensor(_DeviceArray(ptr, n, typestr), device="cuda")


def _copy_from_ptr(dst, ptr: int):
    """dst (contiguous CUDA tensor) <- the device memory at ptr (same size and type)"""
    dst.copy_(device_view(ptr, dst.numel(), dst.dtype))


def _copy_to_ptr(ptr: int, src):
    """the device memory at ptr <- src (contiguous CUDA tensor)"""
    device_view(ptr, src.numel(), src.dtype).copy_(src)


class CoarsePairSet:
    """Normalised (input, target) pairs of one level of the N^3 cube's
    hierarchy: the right-hand sides the level receives in the cycles of
    mixed-precision flexible-CG solves of a Taylor-Green sequence (recorded
    through the level-solver hook, without a graph), with the level's own
    solutions (an exact solve on the level's grid) as targets.  While
    recording, the hook answers with that exact solution, so the recorded
    inputs are those of a cycle whose recursion below the level is exact --
    the cycle the network imitates.  Same normalisation as PairSet: input
    f / rms(f), target x / rms(f) / scale."""

    def __init__(self, N: int, level: int, count: int, seed: int, device=None, skip: int = 0, every: int = 1):
        import torch

        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.N = N >> level  # the level's grid (training and residual loss)
        n = self.N ** 3
        V = (1.0 / self.N) ** 3
        self.inputs = torch.zeros(count, n, dtype=torch.float32, device=dev)
        self.targets = torch.zeros(count, n, dtype=torch.float32, device=dev)
        exact = Context(cube_mesh(self.N), make_options(dict(TARGET_KEYS, precision="fp64", device=dev.index or 0)))
        xe = torch.zeros(n, dtype=torch.float64, device=dev)
        self.count = 0

        def record(stream, rhs, x, shape):
            if shape != (self.N,) * 3:
                raise ValueError(f"level shape {shape}, expected {(self.N,) * 3}")
            torch.cuda.synchronize()  # the recording solve runs without a graph: the rhs is ready
            r = torch.empty(n, dtype=torch.float32, device=dev)
            _copy_from_ptr(r, rhs)
            # the level's system form V b'; the FP32 right-hand side of the
            # singular all-wall system is compatible only to rounding: its
            # mean goes (the solution's mean is free anyway)
            rd = r.double()
            rep = exact.solve((rd - rd.mean()) * V, xe, zero_guess=True)
            if rep.status != 0:
                raise RuntimeError(f"level solve failed: status {rep.status}")
            torch.cuda.synchronize()
            _copy_to_ptr(x, xe.float().contiguous())
            if self.count < count:
                rms = float(torch.sqrt(torch.mean(r.double() ** 2)))
                if rms > 0.0:
                    self.inputs[self.count] = -r / rms
                    self.targets[self.count] = (xe / rms).float()
                    self.count += 1
            torch.cuda.synchronize()

        fine = Context(cube_mesh(N), make_options(dict(TARGET_KEYS, graph="off", device=dev.index or 0)))
        fine.set_level_solver(level, record)
        seq = workloads.TaylorGreenSequence(N, seed, dev)
        for _ in range(skip):
            seq.step()
        xf = torch.zeros(N ** 3, dtype=torch.float64, device=dev)
        while self.count < count:
            rep = fine.solve(seq.rhs(), xf, zero_guess=True)
            if rep.status != 0:
                raise RuntimeError(f"recording solve failed: status {rep.status}")
            for _ in range(every):
                seq.step()
        fine.close()
        exact.close()
        self.scale = float(torch.sqrt(torch.mean(self.targets.double() ** 2)))
        self.targets /= self.scale

    def __len__(self):
        return self.count


class CoarseCorrection:
    """A trained network as the solver of one level of a context's FP32
    cycles (bmg_set_level_solver): the level's right-hand side in, the
    network's solution (scaled back) out, then the level's post-smoothing.

    The network makes the preconditioner nonlinear, and flexible CG can
    stall with it short of the tolerance; ``solve`` therefore gives the
    learned solve ctx's maxIter and, if it has not converged, finishes from
    its x with ``fallback`` -- a context of the same mesh and keys with the
    plain multigrid recursion -- so every solve reaches the tolerance."""

    def __init__(self, net: U.UNet, ctx: Context, level: int, scale: float, fallback: Context | None = None,
                 mode: str = "replace"):
        import torch

        self.net = net
        self.ctx = ctx
        self.level = level
        self.scale = scale
        self.fallback = fallback
        self.fallbacks = 0
        shape = tuple(ctx.shape(level))
        if shape != net.shape:
            raise ValueError(f"network grid {net.shape} is not level {level}'s {shape}")
        # one eager call first: every kernel it queues is loaded before the
        # solver's graph capture calls it
        probe = torch.zeros(net.nvox[0], dtype=torch.float32, device=net.dev)
        net.solve_level(torch.cuda.current_stream().cuda_stream, probe.data_ptr(), probe.data_ptr(), scale)
        torch.cuda.synchronize()
        ctx.set_level_solver(level, self._solve, mode)

    def _solve(self, stream, rhs, x, shape):
        self.net.solve_level(stream, rhs, x, self.scale)

    def solve(self, b, x, zero_guess: bool = True):
        """the learned solve, then (when it stopped short) the plain one from
        its x; returns (report of the last solve, total cycles)"""
        from . import _native as N

        rep = self.ctx.solve(b, x, zero_guess=zero_guess)
        cycles = rep.cycles
        if rep.status == N.NOT_CONVERGED and self.fallback is not None:
            self.fallbacks += 1
            rep = self.fallback.solve(b, x, zero_guess=False)
            cycles += rep.cycles
        return rep, cycles

    def remove(self):
        self.ctx.set_level_solver(self.level, None)


def benchmark_coarse(N: int, level: int, n_pairs: int, steps: int, n_held: int, seed: int = 1,
                     lr: float = 1e-3):
    """The learned coarse-level correction as one measurement: record and
    train on n_pairs level-`level` pairs of one Taylor-Green sequence, then
    time n_held held-out solves of another sequence (mixed precision,
    flexible CG, ||b||-relative 1e-8) with the multigrid recursion below the
    level and with the network in its place.  Returns timings (CUDA events)
    and cycle counts."""
    import time

    import torch

    t0 = time.perf_counter()
    pairs = CoarsePairSet(N, level, n_pairs, seed=seed)
    t_data = time.perf_counter() - t0
    net = U.UNet((pairs.N,) * 3, seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = train(net, pairs, steps, lr=lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    scale = pairs.scale
    del pairs
    torch.cuda.empty_cache()
    keys = dict(TARGET_KEYS, relTol=1e-8)
    plain = Context(cube_mesh(N), make_options(keys))
    stream = torch.cuda.current_stream()
    plain.set_stream(stream.cuda_stream)
    seq = workloads.TaylorGreenSequence(N, seed + 1000, torch.device("cuda", torch.cuda.current_device()))
    for _ in range(17):
        seq.step()
    held = []
    for _ in range(n_held):
        held.append(seq.rhs().clone())
        for _ in range(3):
            seq.step()
    x = torch.zeros(N ** 3, dtype=torch.float64, device=net.dev)
    for q in range(min(3, n_held)):  # warm-up (graph capture)
        plain.solve(held[q], x, zero_guess=True)
    cyc_plain = plain.solve(held[0], x, zero_guess=True).cycles
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    e[0].record(stream)
    cyc0 = [plain.solve(held[q], x, zero_guess=True).cycles for q in range(n_held)]
    e[1].record(stream)
    torch.cuda.synchronize()
    plain_ms = e[0].elapsed_time(e[1]) / n_held
    modes = {}
    for mode in ("replace", "guess"):
        # the learned solve gets twice the plain solve's cycles before the fallback
        learned_ctx = Context(cube_mesh(N), make_options(dict(keys, maxIter=2 * cyc_plain)))
        learned_ctx.set_stream(stream.cuda_stream)
        cc = CoarseCorrection(net, learned_ctx, level, scale, fallback=plain, mode=mode)
        for q in range(min(3, n_held)):
            cc.solve(held[q], x)
        cc.fallbacks = 0
        cyc1, res1 = [], []
        torch.cuda.synchronize()
        e[0].record(stream)
        for q in range(n_held):
            rep, cyc = cc.solve(held[q], x)
            cyc1.append(cyc)
            res1.append(rep.rhs_rel_residual)
        e[1].record(stream)
        torch.cuda.synchronize()
        net.check_errors()
        modes[mode] = {"ms_per_solve": round(e[0].elapsed_time(e[1]) / n_held, 3),
                       "cycles_mean": float(np.mean(cyc1)), "fallbacks": cc.fallbacks,
                       "max_rhs_rel_residual": float(np.max(res1))}
        cc.remove()
        learned_ctx.close()
    # the network alone, once per cycle of the learned solves
    e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    rhs = torch.randn(net.nvox[0], device=net.dev)
    out = torch.empty_like(rhs)
    e2[0].record(stream)
    for _ in range(20):
        net.solve_level(stream.cuda_stream, rhs.data_ptr(), out.data_ptr(), scale)
    e2[1].record(stream)
    torch.cuda.synchronize()
    # the bound for any network: the level solved exactly (eager, cycles only)
    exact_cycles = []
    n_l = (N >> level) ** 3
    V_l = (N >> level) ** -3.0
    exact = Context(cube_mesh(N >> level), make_options(dict(TARGET_KEYS, relTol=1e-10, precision="fp64")))
    bound = Context(cube_mesh(N), make_options(dict(keys, graph="off")))

    def exact_level(stream_, rhs_, x_, shape):
        torch.cuda.synchronize()
        r = device_view(rhs_, n_l).double()
        xe = torch.zeros(n_l, dtype=torch.float64, device=net.dev)
        exact.solve((r - r.mean()) * V_l, xe, zero_guess=True)
        torch.cuda.synchronize()
        device_view(x_, n_l).copy_(xe.float())
        torch.cuda.synchronize()

    bound.set_level_solver(level, exact_level)
    for q in range(min(5, n_held)):
        exact_cycles.append(bound.solve(held[q], x, zero_guess=True).cycles)
    bound.close()
    exact.close()
    plain.close()
    return {"grid": [N] * 3, "level": level, "level_grid": [N >> level] * 3, "training_pairs": n_pairs,
            "training_steps": steps, "held_out": n_held, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
            "final_loss": float(np.mean(losses[-50:])),
            "multigrid_below_level": {"ms_per_solve": round(plain_ms, 3), "cycles_mean": float(np.mean(cyc0))},
            "network_in_place_of_recursion": modes["replace"],
            "network_then_recursion": modes["guess"],
            "network_ms": round(e2[0].elapsed_time(e2[1]) / 20, 3),
            "exact_level_solve_cycles_mean": float(np.mean(exact_cycles))}
