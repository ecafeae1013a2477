"""The coarse end of the V-cycle in one CTA (k_tail_cycle, option
fuseCoarse) against the per-pass launches it replaces: the kernel runs the
same per-item functions (colour_quad_item, restrict_quad_item,
prolong_quad_item, coarse_solve_block), so whole solves are bit-identical in
FP64 and mixed precision, with constant and variable coefficients, with and
without the flexible-CG outer loop, and they launch fewer kernels."""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("krylov", ["none", "fcg"])
@pytest.mark.parametrize("case", ["channel", "sphere"])
@pytest.mark.parametrize("coarse", [0, 1])
def test_tail_cycle_is_bit_identical(native, precision, krylov, case, coarse):
    if case == "channel":
        mesh, b, _ = workloads.channel(64, seed=8)
        lam = None
    else:
        mesh, b, lam = workloads.sphere(64)
    keys = {"relTol": 1e-10, "nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": coarse,
            "precision": precision, "krylov": krylov, "maxIter": 200}
    out = {}
    for fuse in ("on", "off"):
        c = bb.Context(mesh, bb.make_options(dict(keys, fuseCoarse=fuse)))
        if lam is not None:
            c.set_coefficients(lam)
        x = np.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        out[fuse] = (x, rep.cycles, rep.status, rep.kernel_launches)
        c.close()
    assert out["on"][2] == 0 and out["on"][1] == out["off"][1]
    assert np.array_equal(out["on"][0], out["off"][0])
    assert out["on"][3] < out["off"][3]


def test_tail_is_skipped_where_it_does_not_apply(native):
    # W cycles and Jacobi smoothing keep the per-pass launches (same launch count either way)
    mesh, b, _ = workloads.channel(32, seed=9)
    for extra in ({"cycleType": "W"}, {"smoother": "jac"}):
        counts = []
        for fuse in ("on", "off"):
            c = bb.Context(mesh, bb.make_options(dict({"relTol": 1e-8, "coarseLevel": 1, "fuseCoarse": fuse},
                                                      **extra)))
            x = np.zeros_like(b)
            counts.append(c.solve(b, x, zero_guess=True).kernel_launches)
            c.close()
        assert counts[0] == counts[1]
