"""Parity at the benchmarked sizes: the 256³ channel (the bench's headline
workload) and the 256³ two-phase sphere.

* plain FP64 GPU multigrid against the CPU oracle (the restated reference
  multigrid) to 1e-10 relative in the volume-weighted mean-free solution;
* the same GPU solution against the direct GPU FFT solve of the same system
  (an independent FP64 truth for the constant-coefficient channel);
* the headline form (FP32 cycles inside flexible-CG FP64 refinement, 1e-8
  relative residual): its error against the FP64 solution is stated and
  bounded here (1e-6 relative), since it is not an FP64 method.

The oracle solves take tens of seconds on the host cores (all threads).
"""
import os

import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import fft, workloads
from oracle.pyoracle import Oracle
from tests.helpers import rel, vmean

pytestmark = pytest.mark.gpu

V22 = dict(n_pre=2, n_post=2, cycle_type="V", coarse_level=1)
KEYS = {"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": 1, "tolerance": 0}


def _gpu_solve(mesh, b, lam=None, **kw):
    d = dict(KEYS)
    d.update(kw)
    c = bb.Context(mesh, bb.make_options(d))
    if lam is not None:
        c.set_coefficients(lam)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    c.close()
    return x, rep


def _fft_truth(br, b):
    """Laplacian(x) = -f with b = -V f, by the GPU FFT solver."""
    import torch

    dev = torch.device("cuda", 0)
    V = br.cell_volumes().ravel()
    f = torch.from_numpy(-(b / V)).to(dev)
    xf = torch.empty_like(f)
    s = fft.FFTPoissonSolver(br)
    s.solve(xf, f)
    s.close()
    torch.cuda.synchronize()
    return xf.cpu().numpy()


@pytest.fixture(scope="module")
def channel256():
    mesh, b, _ = workloads.channel(256)
    br = mesh.bricks[0]
    x, rep = _gpu_solve(mesh, b, relTol=1e-12, maxIter=200, precision="fp64")
    assert rep.status == 0, rep.status
    return mesh, br, b, x


def test_channel256_fp64_matches_oracle(native, channel256):
    mesh, br, b, x = channel256
    o = Oracle(br.points, periodic=br.periodic, nthreads=os.cpu_count() or 4)
    xo, orep, _, _ = o.solve(b.reshape(br.N), rel_tol=1e-12, max_iter=200, **V22)
    V = br.cell_volumes()
    err = rel(vmean(x.reshape(br.N), V), vmean(xo, V))
    print(f"channel 256^3 FP64 GPU vs oracle: {err:.3e} (oracle {orep.iterations} cycles)")
    assert err <= 1e-10, err


def test_channel256_fp64_matches_fft(native, channel256):
    mesh, br, b, x = channel256
    xf = _fft_truth(br, b)
    V = br.cell_volumes()
    err = rel(vmean(x.reshape(br.N), V), vmean(xf.reshape(br.N), V))
    print(f"channel 256^3 FP64 GPU multigrid vs GPU FFT solver: {err:.3e}")
    assert err <= 1e-10, err


def test_channel256_headline_error_vs_fp64(native, channel256):
    """The benchmarked method (mixed precision + flexible CG to 1e-8): the
    error of its solution against the FP64 solution, stated."""
    mesh, br, b, x = channel256
    xm, rep = _gpu_solve(mesh, b, relTol=1e-8, precision="mixed", krylov="fcg", criterion="rhs")
    assert rep.status == 0 and rep.rel_residual <= 1e-8
    xf = _fft_truth(br, b)
    V = br.cell_volumes()
    err = rel(vmean(xm.reshape(br.N), V), vmean(xf.reshape(br.N), V))
    print(f"channel 256^3 mixed+FCG (1e-8) vs FP64 FFT solution: {err:.3e}")
    assert err <= 1e-6, err


def test_sphere256_fp64_matches_oracle(native):
    """The two-phase variable coefficient (density ratio 1000) at 256³."""
    mesh, b, lam = workloads.sphere(256)
    br = mesh.bricks[0]
    x, rep = _gpu_solve(mesh, b, lam=lam, relTol=1e-12, maxIter=400, precision="fp64")
    assert rep.status == 0, rep.status
    o = Oracle(br.points, periodic=br.periodic, nthreads=os.cpu_count() or 4)
    o.set_lambda(*lam)
    xo, orep, _, _ = o.solve(b.reshape(br.N), rel_tol=1e-12, max_iter=400, **V22)
    V = br.cell_volumes()
    err = rel(vmean(x.reshape(br.N), V), vmean(xo, V))
    print(f"sphere 256^3 FP64 GPU vs oracle: {err:.3e} (GPU {rep.cycles}, oracle {orep.iterations} cycles)")
    assert err <= 1e-10, err
    xm, repm = _gpu_solve(mesh, b, lam=lam, relTol=1e-8, maxIter=400, precision="mixed", krylov="fcg",
                          criterion="rhs")
    assert repm.status == 0 and repm.rel_residual <= 1e-8
    errm = rel(vmean(xm.reshape(br.N), V), vmean(xo, V))
    print(f"sphere 256^3 mixed+FCG (1e-8) vs FP64 oracle solution: {errm:.3e}")
    assert errm <= 1e-5, errm
