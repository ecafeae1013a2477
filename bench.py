#!/usr/bin/env python
"""Benchmark of the B200 multigrid Poisson solve.

Workload: the 256^3 channel (periodic x and z, tanh-clustered walls in y,
gamma = 2; seeded divergence RHS plus a sin(2 pi x) cos(pi y) mode), solved
to 1e-8 relative residual, V(2,2), red-black Gauss-Seidel, coarsest 4^3
direct.  One step = one complete solve from a zero initial guess.

value      ms per solve of the headline method (FP32 V-cycles as the
           preconditioner of a flexible-CG loop in FP64), device-resident
           inputs, CUDA events.  The reference's plain FP64 loop and the two
           intermediate forms are timed beside it (arms_ms_per_solve).
e2e        the same through the reference-facing plugin call
           (GPUMG.solve on pinned host arrays: host->device copy of b and
           device->host copy of x inside the timed region).
roofline   the level-0 red-black pass of the headline path, achieved
           algorithmic GB/s against the measured HBM copy bandwidth.
cpu_baseline / --impl reference
           the CPU restatement of the reference multigrid (oracle/, "port"),
           one full solve of the same workload on the host cores.

Multi-GPU: the solve does not shard (one brick on one GPU); with --gpus N
each rank runs an independent replica and value is the job's time per
solve (max over ranks of the timed region / (N * steps)).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/solve to 1e-8 rel residual @256^3: learned+mixed vs plain GPU MG; HBM GB/s"
SOLVER_KEYS = {"relTol": 1e-8, "tolerance": 0, "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2,
               "coarseLevel": 1, "smoother": "rbgs"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock and throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def _lines(self):
        with open(self.path) as f:
            return f.readlines()

    def mark(self) -> None:
        """Start of the timed region: later samples count."""
        if self.proc is not None:
            time.sleep(1.0)  # nvidia-smi takes a moment to begin sampling
            self.first = len(self._lines())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self._lines()[getattr(self, "first", 0):]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(N: int, steps: int | None = None, warmup: int = 0, stale: int = 1,
                  nthreads: int | None = None):
    """Time the oracle (CPU restatement of the reference MG) on the benchmark
    workload: full solves from a zero guess.  nthreads threads (default: all
    host threads) emulate as many ranks of a slab decomposition of the brick
    (P, 1, 1): each owns a contiguous range of i-planes in every pass, with a
    barrier between passes where the reference exchanges halos, and levels
    with fewer than 2P planes run on one thread, as the reference gathers
    its coarse levels.  stale: the reference's stale finest-level residual
    on the first repetition (MG.C:72), on (1, the reference) or off (0)."""
    from briscola_b200 import workloads
    from oracle.pyoracle import Oracle

    mesh, b, _ = workloads.channel(N)
    br = mesh.bricks[0]
    threads = nthreads or os.cpu_count() or 1
    o = Oracle(br.points, periodic=br.periodic, nthreads=threads)
    bb = b.reshape(br.N)
    kw = dict(rel_tol=1e-8, abs_tol=0.0, n_pre=2, n_post=2, cycle_type="V", coarse_level=1,
              stale_residual=stale)
    times, cycles = [], 0
    for s in range(warmup + (steps or 1)):
        t = time.perf_counter()
        x, rep, hist, rc = o.solve(bb, **kw)
        dt = (time.perf_counter() - t) * 1e3
        cycles = rep.iterations
        if s >= warmup:
            times.append(dt)
    return times, cycles, threads


def cpu_one_core(N: int, cycles: int):
    """One core (one reference rank owning the whole brick), a bounded
    sample: a solve stopped after 1 cycle and one stopped after 3 give the
    set-up cost and the cost of a cycle; ms per solve = set-up + cycles
    times the cycle cost."""
    from briscola_b200 import workloads
    from oracle.pyoracle import Oracle

    mesh, b, _ = workloads.channel(N)
    br = mesh.bricks[0]
    o = Oracle(br.points, periodic=br.periodic, nthreads=1)
    bb = b.reshape(br.N)
    kw = dict(rel_tol=0.0, abs_tol=0.0, n_pre=2, n_post=2, cycle_type="V", coarse_level=1)
    t = {}
    for m in (1, 3):
        t0 = time.perf_counter()
        o.solve(bb, max_iter=m, **kw)
        t[m] = (time.perf_counter() - t0) * 1e3
    per_cycle = (t[3] - t[1]) / 2
    setup = max(t[1] - per_cycle, 0.0)
    return setup + cycles * per_cycle, per_cycle, setup


def max_over_ranks(value: float, dist, device) -> float:
    """The slowest rank's time: replicas (one independent solve per rank, no
    collective on the data path) are timed together and the job is as fast
    as its slowest rank.  dist is torch.distributed (NCCL on the GPUs, gloo
    in the CPU tests) or None for one rank."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    times, cycles, threads = cpu_reference(args.size, steps=args.steps, warmup=args.warmup)
    v = sum(times) / len(times)
    sample = f"{args.steps} full solves of the {args.size}^3 channel, {cycles} V(2,2) cycles each"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ms/solve",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args),
        "cpu_baseline": {"value": round(v, 3), "unit": "ms/solve", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(v, 3), "unit": "ms/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"channel {args.size}^3 (periodic x,z; tanh gamma=2 walls in y), seeded "
                        "div(N(0,1) velocity) + sin(2 pi x)cos(pi y) RHS, zero mean",
            "grid": [args.size] * 3, "solver": "V(2,2) RBGS, linear transfers, coarsest 4^3 direct",
            "stop": "1e-8 relative residual (FP64-checked)",
            "precision": "fp32 cycles as preconditioner of flexible-CG fp64 refinement",
            "l2_flush": "inputs and hierarchy larger than L2 (x, b 134 MB each at 256^3)",
            "parallelism": "replicas" if args.gpus > 1 else "single GPU"}


def tuning_string(c):
    """The autotuner's smoother launch shapes, level:precision:stages:chunk
    (stages 0: pass by pass), in the form --tuning takes."""
    out = []
    for lvl in range(c.num_levels):
        for prec in (0, 1):
            stages, chunk = c.tuning(lvl, prec)
            out.append(f"{lvl}:{prec}:{stages}:{chunk or 64}")
    return ",".join(out)


def profile_region(args, local):
    """One headline solve (or one U-Net forward at the bench size) after
    set-up and warm-up, bracketed by the CUDA profiler API."""
    import torch

    import briscola_b200 as bb
    from briscola_b200 import workloads

    stream = torch.cuda.current_stream()
    if args.profile_region in ("fft", "fft_box"):
        from briscola_b200 import fft

        mesh, _, _ = (workloads.channel if args.profile_region == "fft" else workloads.cavity)(args.size)
        solver = fft.FFTPoissonSolver(mesh.bricks[0], device=local)
        f = torch.randn(mesh.bricks[0].N, dtype=torch.float64, device=f"cuda:{local}")
        x = torch.empty_like(f)
        for _ in range(args.warmup):
            solver.solve(x, f)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        solver.solve(x, f)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        solver.close()
        return
    if args.profile_region == "unet_fwd":
        from briscola_b200 import unet

        net = unet.UNet((args.size,) * 3)
        x = torch.randn(args.size ** 3, device=f"cuda:{local}")
        for _ in range(args.warmup):
            net.forward(x)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        net.forward(x)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        net.check_errors()
        return
    kw = dict(precision="fp64")
    if args.profile_region.startswith("mixed_fcg"):
        kw = dict(precision="mixed", krylov="fcg")
    if args.profile_region == "mixed_fcg_fused":
        kw.update(autotune="off")  # the fused smoother on every level it fits (3 stages, 64-plane chunks)
    mesh, b, _ = workloads.channel(args.size)
    if args.profile_region == "multibrick":
        # the seven-brick mesh's mixed flexible-CG solve
        kw = dict(precision="mixed", krylov="fcg", coarseLevel=0)
        mesh, b, _ = workloads.multibrick(1)
    # the same kernels launched one by one (the profiler cannot see into a
    # graph with a conditional loop)
    if args.tuning:
        kw.update(autotune="off")
    c = bb.Context(mesh, bb.make_options(dict(SOLVER_KEYS, device=local, graph="off", **kw)))
    c.set_stream(stream.cuda_stream)
    if args.tuning:
        for item in args.tuning.split(","):
            lvl, prec, stages, chunk = (int(v) for v in item.split(":"))
            c.set_tuning(lvl, prec, stages, chunk)
    b_d = torch.from_numpy(b).to(f"cuda:{local}")
    x_d = torch.zeros_like(b_d)
    for _ in range(args.warmup):
        c.solve(b_d, x_d, zero_guess=True)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    rep = c.solve(b_d, x_d, zero_guess=True)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    if rep.status != 0:
        raise RuntimeError(f"solve failed: status {rep.status}")


def _fft_one(args, local, stream, br, barrier):
    """Solves of one brick (device-resident, CUDA events) and the max of the
    discrete Laplacian residual over max |f|."""
    import torch

    from briscola_b200 import fft

    solver = fft.FFTPoissonSolver(br, device=local)
    n = br.N
    g = torch.Generator(device=f"cuda:{local}").manual_seed(11)
    f = torch.randn(n, dtype=torch.float64, device=f"cuda:{local}", generator=g)
    # a compatible right-hand side for the walled problem: volume-weighted mean zero
    V = torch.from_numpy(br.cell_volumes()).to(f.device)
    f -= (f * V).sum() / V.sum()
    x = torch.empty_like(f)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        solver.solve(x, f)
    barrier()
    reps = max(10, args.steps * 4)
    e0.record(stream)
    for _ in range(reps):
        solver.solve(x, f)
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1) / reps
    # residual of the cell-centred Laplacian (periodic axes wrap, zero-gradient
    # walls: mirrored ghost cells)
    h = [torch.from_numpy(br.cell_sizes(d)).to(f.device) for d in range(3)]
    r = f.clone()
    for d in range(3):
        hd = h[d]
        if br.periodic[d]:
            hg = torch.cat([hd[-1:], hd, hd[:1]])
            xm, xp = torch.roll(x, 1, d), torch.roll(x, -1, d)
        else:
            hg = torch.cat([hd[:1], hd, hd[-1:]])
            idx = torch.arange(n[d], device=f.device)
            xm = x.index_select(d, (idx - 1).clamp(min=0))
            xp = x.index_select(d, (idx + 1).clamp(max=n[d] - 1))
        hc = hg[1:-1]
        dw = (hg[1:-1] + hg[:-2]) / 2
        de = (hg[1:-1] + hg[2:]) / 2
        shape = [1, 1, 1]
        shape[d] = -1
        hc, dw, de = hc.view(shape), dw.view(shape), de.view(shape)
        r += (xm - x) / (dw * hc) + (xp - x) / (de * hc)
    res = float(r.abs().max() / f.abs().max())
    cells = n[0] * n[1] * n[2]
    sdir = solver.solve_direction
    solver.close()
    return {"ms_per_solve": round(ms, 4), "solve_direction": sdir, "max_residual_over_max_rhs": res,
            "algorithmic_gb_per_s": round(cells * 8 * 10 / (ms * 1e-3) / 1e9, 1)}


def fft_timing(args, local, stream, mesh, barrier):
    """The FFT Poisson solver (briscola_b200.fft) on the bench's channel (real
    FFTs along x and z) and on the closed box of the same size (all walls
    zero-gradient: cosine transforms along both transform axes):
    Laplacian(x) = -f for a seeded zero-mean f, device-resident, CUDA events;
    the discrete Laplacian residual is checked on the device."""
    from briscola_b200 import workloads

    out = {"workload": "the bench channel, Laplacian(x) = -f, seeded N(0,1) f with zero volume-weighted mean"}
    out.update(_fft_one(args, local, stream, mesh.bricks[0], barrier))
    out["algorithmic_bytes_note"] = ("10 passes of 8 B/cell: read+write per transform (4) and "
                                     "tridiagonal (read+write each way)")
    box, _, _ = workloads.cavity(args.size)
    out["closed_box"] = dict({"workload": f"uniform {args.size}^3 box, all walls zero-gradient (REDFT10/01 "
                                          "along both transform axes)"},
                             **_fft_one(args, local, stream, box.bricks[0], barrier))
    return out


def split_timing(args, local, stream, barrier):
    """The split Poisson solver (briscola_b200.split) on the two-phase sphere
    coefficient: corrections on the GPU FFT solver, with and without the GPU
    multigrid as preconditioner; the residual of -div(lambda grad x) = f is
    evaluated on the device."""
    import numpy as np
    import torch

    from briscola_b200 import split, workloads

    mesh, _, lam = workloads.sphere(args.size)
    br = mesh.bricks[0]
    dev = torch.device("cuda", local)
    lamd = [torch.from_numpy(np.ascontiguousarray(l)).to(dev) for l in lam]
    g = torch.Generator(device=dev).manual_seed(12)
    f = torch.randn(br.N, dtype=torch.float64, device=dev, generator=g)
    f -= f.mean()  # uniform cells: a compatible right-hand side for the walled box
    h = [torch.from_numpy(br.cell_sizes(d)).to(dev) for d in range(3)]

    def residual(x):
        # -div(lambda grad x) - f with zero-gradient walls (no flux through them)
        div = torch.zeros_like(x)
        for d in range(3):
            n = br.N[d]
            dx = torch.diff(x, dim=d)  # x[q+1] - x[q] at the n-1 interior faces
            hc = h[d]
            dist = 0.5 * (hc[1:] + hc[:-1])
            shape = [1, 1, 1]
            shape[d] = -1
            lf = lamd[d].narrow(d, 1, n - 1)
            flux = lf * dx / dist.view(shape)
            zero = torch.zeros_like(flux.narrow(d, 0, 1))
            fp = torch.cat([zero, flux, zero], dim=d)  # flux through face q (0..n)
            div += (fp.narrow(d, 1, n) - fp.narrow(d, 0, n)) / hc.view(shape)
        r = -div - f
        return float(r.abs().max() / f.abs().max())

    out = {"workload": f"sphere {args.size}^3 coefficient (rho 1 / 1000), all walls, seeded N(0,1) zero-mean f, "
                       "-div(lambda grad x) = f from x = 0"}
    arms = (("fft_only_ncorr4", {"nCorr": 4}),
            ("mg_preconditioned_ncorr2", {"nCorr": 2, "preconditioner": {
                "type": "GPUMG", "precision": "mixed", "krylov": "fcg", "maxIter": 4, "relTol": 0, "tolerance": 0,
                "cycleType": "V", "nSweepsPre": 2, "nSweepsPost": 2, "coarseLevel": 1}}))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for name, extra in arms:
        s = split.SplitPoissonSolver(mesh, dict({"solver": {"type": "FFT"}, "prediction": "off"}, **extra),
                                     device=local)
        x = torch.zeros_like(f)
        s.solve(x, f, lamd)  # warm-up; sets the preconditioner's coefficients
        reps = 3
        barrier()
        e0.record(stream)
        for _ in range(reps):
            x.zero_()
            s.solve(x, f, lamd, constMatrix=True)
        e1.record(stream)
        barrier()
        out[name] = {"ms_per_solve": round(e0.elapsed_time(e1) / reps, 3),
                     "max_residual_over_max_rhs": residual(x)}
        s.close()
    return out


def unet_timing(args, local, stream):
    """U-Net forward at the bench size (algorithmic TFLOP/s of the 3x3x3
    convolutions) and one training step at half the size."""
    import torch

    from briscola_b200 import unet

    out = {}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for size, what in ((args.size, "forward"), (args.size // 2, "train_step")):
        net = unet.UNet((size,) * 3)
        x = torch.randn(size ** 3, device=f"cuda:{local}")
        t = torch.randn(size ** 3, device=f"cuda:{local}")
        run = (lambda: net.forward(x)) if what == "forward" else (lambda: net.train_step(x, t, lr=1e-4))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        reps = 10
        e0.record(stream)
        for _ in range(reps):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        net.check_errors()
        ms = e0.elapsed_time(e1) / reps
        flops = unet.forward_flops((size,) * 3) * (1 if what == "forward" else 3)
        out[what] = {"grid": [size] * 3, "ms": round(ms, 3), "tflops_algorithmic": round(flops / ms / 1e9, 1)}
        del net
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-multibrick", action="store_true")
    ap.add_argument("--no-unet", action="store_true")
    ap.add_argument("--no-variable", action="store_true")
    ap.add_argument("--no-fft", action="store_true")
    ap.add_argument("--no-split", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--learned-size", type=int, default=128)
    ap.add_argument("--learned-pairs", type=int, default=2000)
    ap.add_argument("--learned-steps", type=int, default=2000)
    ap.add_argument("--learned-held", type=int, default=200)
    ap.add_argument("--no-learned-coarse", action="store_true")
    ap.add_argument("--profile-region", choices=["mixed_fcg", "mixed_fcg_fused", "fp64", "unet_fwd", "fft", "fft_box",
                                                         "multibrick"],
                    default=None,
                    help="set up, warm up, then run one solve (or one U-Net forward) between "
                         "cudaProfilerStart/Stop for ncu --profile-from-start off; prints no bench line")
    ap.add_argument("--tuning", default=None,
                    help="with --profile-region: smoother launch shapes to pin instead of autotuning "
                         "(level:precision:stages:chunk,...; the bench line's 'tuning' field), since "
                         "the profiler's per-launch overhead skews the autotuner's timings")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import briscola_b200 as bb
    from briscola_b200 import workloads

    if args.profile_region:
        profile_region(args, local)
        return

    mesh, b, _ = workloads.channel(args.size)
    n = b.size
    stream = torch.cuda.current_stream()
    # the headline method, the reference's plain FP64 loop and the two
    # intermediate forms (one change each)
    ARMS = {"mixed_fcg": dict(precision="mixed", krylov="fcg"), "fp64": dict(precision="fp64", krylov="none"),
            "mixed": dict(precision="mixed", krylov="none"), "fp64_fcg": dict(precision="fp64", krylov="fcg")}
    ctx = {}
    for arm, kw in ARMS.items():
        ctx[arm] = bb.Context(mesh, bb.make_options(dict(SOLVER_KEYS, device=local, **kw)))
        ctx[arm].set_stream(stream.cuda_stream)
    b_d = torch.from_numpy(b).to(f"cuda:{local}")
    x_d = torch.zeros_like(b_d)

    def solve(prec):
        rep = ctx[prec].solve(b_d, x_d, zero_guess=True)
        if rep.status != 0:
            raise RuntimeError(f"solve failed: status {rep.status}")
        return rep

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(prec, steps):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        launches, cycles = 0, []
        e0.record(stream)
        for _ in range(steps):
            rep = solve(prec)
            launches += rep.kernel_launches
            cycles.append(rep.cycles)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
        return ms, launches, cycles

    clk = Clocks(local)
    clk.start()
    for _ in range(args.warmup):
        for arm in ARMS:
            solve(arm)
    clk.mark()
    ms_head, launches, cyc_head = timed("mixed_fcg", args.steps)
    clocks = clk.stop()
    ms_fp64, _, cyc_fp64 = timed("fp64", args.steps)
    ms_mixed, _, cyc_mixed = timed("mixed", args.steps)
    ms_fp64_fcg, _, cyc_fp64_fcg = timed("fp64_fcg", args.steps)
    rep_head = solve("mixed_fcg")
    per_solve = ms_head / (args.steps * world)

    # ---- roofline of the dominant kernel: the level-0 fused smoothing step
    # (FP32, V(2,2): two sweeps = 5 colour stages in one launch) ----
    c = ctx["mixed_fcg"]
    reps = 30
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    pass_ms = []
    for r in range(reps):
        e0.record(stream)
        c.smooth(0, SOLVER_KEYS["nSweepsPost"], precision=1)
        e1.record(stream)
        torch.cuda.synchronize()
        pass_ms.append(e0.elapsed_time(e1))
    # the step's colour stages (5 for two sweeps) go in launches of S stages
    stages_per_launch, chunk = c.tuning(0, 1)
    n_stages = 5 if SOLVER_KEYS["nSweepsPost"] == 2 else 3 * SOLVER_KEYS["nSweepsPost"]
    launches_per_step = -(-n_stages // max(stages_per_launch, 1))
    t_pass = statistics.median(pass_ms) * 1e-3 / launches_per_step
    cells = n
    # FP32 algorithmic bytes per launch: a single colour pass needs half a
    # sweep's read x, read b, write x (6 B/cell); a fused launch of two or
    # more stages needs a whole one (12 B/cell)
    alg_bytes = (12.0 if stages_per_launch >= 2 else 6.0) * cells
    hbm, peak_kind = peaks()
    achieved = alg_bytes / t_pass / 1e9
    # level 0 is kept in parity-split rows (rowLayout split, n2 % 16 == 0):
    # its colour passes run k_colour_split
    n2_0 = c.shape(0)[2]
    split0 = n2_0 % 16 == 0 and not stages_per_launch
    pass_kernel = "k_colour_split" if split0 else "k_colour_quad"
    # DRAM bytes per launch from the committed ncu summary of this kernel
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_sweep_fp32_channel256.md" if stages_per_launch else
                      f"{pass_kernel}_fp32_channel256.md")
    if os.path.exists(tp):
        import re

        m = re.search(r"^traffic per launch \(bytes\): ([0-9.e+]+)", open(tp).read(), re.M)
        traffic = float(m.group(1)) if m else None

    # ---- the same for the plain FP64 path's level-0 smoothing step ----
    c64 = ctx["fp64"]
    pass64 = []
    for r in range(reps):
        e0.record(stream)
        c64.smooth(0, SOLVER_KEYS["nSweepsPost"], precision=0)
        e1.record(stream)
        torch.cuda.synchronize()
        pass64.append(e0.elapsed_time(e1))
    st64, chunk64 = c64.tuning(0, 0)
    lps64 = -(-n_stages // max(st64, 1))
    t64 = statistics.median(pass64) * 1e-3 / lps64
    alg64 = (24.0 if st64 >= 2 else 12.0) * cells
    ach64 = alg64 / t64 / 1e9
    traffic64 = None
    tp64 = os.path.join(ROOT, "profiles", f"{pass_kernel}_fp64_channel256.md")
    if not st64 and os.path.exists(tp64):
        import re

        m = re.search(r"^traffic per launch \(bytes\): ([0-9.e+]+)", open(tp64).read(), re.M)
        traffic64 = float(m.group(1)) if m else None
    roof64 = {"bound": "hbm", "kernel": (f"k_sweep<double> level 0 ({lps64} launches of up to {st64} colour "
                                         f"stages, {chunk64}-plane chunks)" if st64 else
                                         f"{pass_kernel}<double> level 0 ({lps64} passes per 2-sweep step)"),
              "traffic": traffic64,
              "achieved": round(ach64, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach64 / hbm, 4),
              "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg64,
              "launch_us": round(t64 * 1e6, 2)}

    # ---- the headline solution's error against an FP64 solution of the same
    # system: the direct GPU FFT solve (Laplacian(x) = -f, b = -V f) ----
    from briscola_b200 import fft as _fft

    br0 = mesh.bricks[0]
    Vd = torch.from_numpy(br0.cell_volumes().ravel()).to(f"cuda:{local}")
    solve("mixed_fcg")
    xf = torch.empty_like(b_d)
    fs = _fft.FFTPoissonSolver(br0, device=local)
    fs.solve(xf, -(b_d / Vd))
    fs.close()

    def _centred(t):
        return t - (t * Vd).sum() / Vd.sum()

    err_fp64 = float(torch.linalg.norm(_centred(x_d) - _centred(xf)) / torch.linalg.norm(_centred(xf)))
    del xf, Vd

    # ---- end to end through the plugin call with host buffers ----
    d = bb.Dictionary(dict(SOLVER_KEYS, type="GPUMG", precision="mixed", krylov="fcg", device=local))
    s = bb.solver.New(d, mesh)
    s.context.set_stream(stream.cuda_stream)
    bh = torch.from_numpy(b).pin_memory()
    xh = torch.zeros(n, dtype=torch.float64).pin_memory()
    sys_ = bb.LinearSystem(mesh, xh.numpy(), bh.numpy(), zero_guess=True)
    import contextlib
    import io

    with contextlib.redirect_stdout(io.StringIO()):
        for _ in range(2):
            s.solve(sys_)
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            s.solve(sys_)
        e1.record(stream)
        barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, f"cuda:{local}") / world

    # ---- the seven-brick mesh (2.55 M cells, one launch per level across
    # bricks, ghost exchange on the device): FP64 and mixed ms per solve ----
    multibrick = None
    if not args.no_multibrick:
        mb_mesh, mb_b, _ = workloads.multibrick(1)
        mb_bd = torch.from_numpy(mb_b).to(f"cuda:{local}")
        mb_x = torch.zeros_like(mb_bd)
        multibrick = {"workload": "7 bricks (128x64x64, 96x96x96, 64x128x32, 128x32x64, 64x64x64, "
                                  "48x96x48, 32x32x128), h = 1/128, Neumann walls, N(0,1) zero-mean RHS, "
                                  "V(2,2), coarsest level (622 cells) direct, 1e-8",
                      "cells": int(mb_b.size)}
        for prec in ("fp64", "mixed", "mixed_fcg"):
            kw = dict(precision="mixed", krylov="fcg") if prec == "mixed_fcg" else dict(precision=prec)
            cm = bb.Context(mb_mesh, bb.make_options(dict(SOLVER_KEYS, coarseLevel=0, device=local, **kw)))
            cm.set_stream(stream.cuda_stream)
            for _ in range(3):
                cm.solve(mb_bd, mb_x, zero_guess=True)
            barrier()
            e0.record(stream)
            for _ in range(args.steps):
                rep = cm.solve(mb_bd, mb_x, zero_guess=True)
            e1.record(stream)
            barrier()
            if rep.status != 0:
                raise RuntimeError(f"seven-brick solve failed: status {rep.status}")
            multibrick[prec] = {"ms_per_solve": round(e0.elapsed_time(e1) / args.steps, 4),
                                "cycles": rep.cycles, "rel_residual": rep.rel_residual}
            cm.close()
        del mb_bd, mb_x

    unet_t = None if args.no_unet else unet_timing(args, local, stream)

    # ---- two-phase variable coefficient (sphere, density ratio 1000) ----
    variable = None
    if not args.no_variable:
        vmesh, vb, vlam = workloads.sphere(args.size)
        vbd = torch.from_numpy(vb).to(f"cuda:{local}")
        vx = torch.zeros_like(vbd)
        variable = {"workload": f"sphere {args.size}^3, all walls, rho 1 / 1000 (radius 0.2, seeded centre), "
                                "VOF ramp over 2 cells, face coefficient mean of 1/rho, N(0,1) zero-mean RHS, 1e-8"}
        for arm, kw in (("fp64", dict(precision="fp64")), ("mixed_fcg", dict(precision="mixed", krylov="fcg"))):
            cv = bb.Context(vmesh, bb.make_options(dict(SOLVER_KEYS, device=local, maxIter=2000, **kw)))
            cv.set_stream(stream.cuda_stream)
            cv.set_coefficients(vlam)
            for _ in range(2):
                cv.solve(vbd, vx, zero_guess=True)
            barrier()
            e0.record(stream)
            nrep = max(1, args.steps // 2)
            for _ in range(nrep):
                rep = cv.solve(vbd, vx, zero_guess=True)
            e1.record(stream)
            barrier()
            variable[arm] = {"ms_per_solve": round(e0.elapsed_time(e1) / nrep, 3), "cycles": rep.cycles,
                             "status": rep.status, "rel_residual": rep.rel_residual}
            cv.close()
        del vbd, vx

    # ---- FFT Poisson solver on the same channel (periodic x, z; walls in y) ----
    fft_t = None
    if not args.no_fft:
        fft_t = fft_timing(args, local, stream, mesh, barrier)

    split_t = None
    if not args.no_split:
        split_t = split_timing(args, local, stream, barrier)

    # ---- learned initial guess (config 5) ----
    learned_t = None
    if not args.no_learned:
        from briscola_b200 import learned

        learned_t = learned.benchmark(args.learned_size, args.learned_pairs, args.learned_steps,
                                      args.learned_held)
        torch.cuda.empty_cache()

    # ---- learned coarse-level correction (config 5): the network on the 64^3
    # level of the 128^3 and of the 256^3 cube in place of the recursion below ----
    learned_coarse = None
    if not args.no_learned_coarse:
        from briscola_b200 import learned

        learned_coarse = []
        for N in sorted({128, args.size}):
            level = {128: 1, 256: 2, 512: 3}.get(N)
            if level is None:
                continue
            learned_coarse.append(learned.benchmark_coarse(N, level, args.learned_pairs, args.learned_steps,
                                                           args.learned_held))
            torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        times, cycles, threads = cpu_reference(args.size, steps=1)
        times_ns, cycles_ns, _ = cpu_reference(args.size, steps=1, stale=0)
        one_ms, one_cycle_ms, one_setup_ms = cpu_one_core(args.size, cycles)
        cpu = {"value": round(times[0], 1), "unit": "ms/solve", "cores": threads, "kind": "port",
               "ranks": threads, "decomposition": [threads, 1, 1],
               "sample": f"one full solve of the same {args.size}^3 workload by the CPU restatement "
                         f"of the reference MG ({cycles} V(2,2) cycles) on {threads} threads emulating "
                         f"{threads} ranks of a ({threads},1,1) slab decomposition (contiguous i-plane "
                         "ranges, a barrier per pass for the halo exchange, coarse levels gathered to one "
                         "thread); stale finest-level residual of MG.C:72 on, as in the reference",
               "stale_residual_off": {"value": round(times_ns[0], 1), "cycles": cycles_ns},
               "one_core": {"value": round(one_ms, 1), "ranks": 1, "decomposition": [1, 1, 1],
                            "ms_per_cycle": round(one_cycle_ms, 1), "setup_ms": round(one_setup_ms, 1),
                            "sample": "solves stopped after 1 and after 3 cycles on one thread; "
                                      f"value = set-up + {cycles} cycles"}}

    # algorithmic bytes of one FP64 V(2,2) cycle: 164.6 B per finest cell
    hbm_gbs_fp64 = 164.6 * cells * statistics.mean(cyc_fp64) / (ms_fp64 / args.steps * 1e-3) / 1e9

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(per_solve, 4), "unit": "ms/solve", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_head / args.steps, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": workload_config(args),
            "method": "FP32 V(2,2) cycles as the preconditioner of a flexible-CG FP64 refinement loop "
                      "(FP64 residual, update, coarse solve and mean removal); learned guess not in this line",
            "plain_fp64_ms_per_solve": round(ms_fp64 / (args.steps * world), 4),
            "speedup_vs_plain_fp64": round(ms_fp64 / ms_head, 3),
            "arms_ms_per_solve": {"mixed_fcg": round(ms_head / (args.steps * world), 4),
                                  "fp64 (reference loop)": round(ms_fp64 / (args.steps * world), 4),
                                  "mixed (reference loop)": round(ms_mixed / (args.steps * world), 4),
                                  "fp64_fcg": round(ms_fp64_fcg / (args.steps * world), 4)},
            "arms_cycles": {"mixed_fcg": cyc_head[0], "fp64": cyc_fp64[0], "mixed": cyc_mixed[0],
                            "fp64_fcg": cyc_fp64_fcg[0]},
            "rel_residual": rep_head.rel_residual,
            "error_vs_fp64": {"value": err_fp64, "against": "the direct FP64 GPU FFT solve of the same system",
                              "norm": "relative L2 of the volume-weighted mean-free solutions"},
            "roofline_fp64_smoother": roof64,
            "hbm_gbs_fp64_cycle_algorithmic": round(hbm_gbs_fp64, 1),
            "roofline": {"bound": "hbm",
                         "kernel": (f"k_sweep<float> level 0 ({launches_per_step} launches of up to "
                                    f"{stages_per_launch} colour stages per 2-sweep step, {chunk}-plane chunks)"
                                    if stages_per_launch else
                                    f"{pass_kernel}<float> level 0 ({launches_per_step} passes per "
                                    "2-sweep step)"),
                         "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                         "launch_us": round(t_pass * 1e6, 2)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_ms, 4), "unit": "ms/solve", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * n},
            "gpu_launches": launches, "clocks": clocks,
            "tuning": tuning_string(ctx["mixed_fcg"]),
            "multibrick": multibrick,
            "unet": unet_t,
            "variable_coefficient": variable,
            "fft": fft_t,
            "split": split_t,
            "learned": learned_t,
            "learned_coarse": learned_coarse,
        }
        print(json.dumps(line), flush=True)
    for cc in ctx.values():
        cc.close()
    s.context.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
