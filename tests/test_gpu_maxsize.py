"""The largest brick both GPU solvers take: the 512³ channel (134 M cells;
the FFT solver transforms powers of two up to 512).  The multigrid (mixed
precision, flexible CG) and the direct FFT solve of the same system agree,
and the multigrid's 32-bit slab indexing holds at this size."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import fft, workloads

pytestmark = pytest.mark.gpu


def test_512_channel_matches_the_fft_solver(native):
    torch = pytest.importorskip("torch")
    mesh, b, _ = workloads.channel(512)
    br = mesh.bricks[0]
    dev = torch.device("cuda", 0)
    V = torch.from_numpy(br.cell_volumes().ravel()).to(dev)
    bd = torch.from_numpy(b).to(dev)
    del b
    x = torch.zeros_like(bd)
    c = bb.Context(mesh, bb.make_options({"relTol": 1e-12, "tolerance": 0, "cycleType": "V", "nSweepsPre": 2,
                                          "nSweepsPost": 2, "coarseLevel": 1, "precision": "mixed",
                                          "krylov": "fcg", "maxIter": 100, "autotune": "off"}))
    rep = c.solve(bd, x, zero_guess=True)
    c.close()
    assert rep.status == 0, rep.status
    assert rep.rel_residual <= 1e-11
    # Laplacian(x) = -f with b = -V f
    f = -(bd / V)
    xf = torch.empty_like(f)
    s = fft.FFTPoissonSolver(br)
    s.solve(xf, f)
    s.close()
    torch.cuda.synchronize()

    def centred(t):
        return t - (t * V).sum() / V.sum()

    err = torch.linalg.norm(centred(x) - centred(xf)) / torch.linalg.norm(centred(xf))
    assert float(err) <= 1e-8, float(err)
