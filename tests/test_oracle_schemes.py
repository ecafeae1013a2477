"""The oracle's other cycle options, pinned to the reference's formulas on
the CPU: the average restriction (averageRestrictionScheme.C:35-77: the
children's mean of r/V times the coarse volume), injection
(injectionProlongationScheme.C:14-33: the parent's value), and coarseMode
smooth on a singular system (the pinned coarse matrix of solver.C:201-231:
the first cell held at zero)."""
import numpy as np
import pytest

from briscola_b200.mesh import geometric_points, uniform_points
from oracle.pyoracle import Oracle

PTS = [uniform_points(16), geometric_points(8, 2.0), geometric_points(12, 0.5)]


def _children_mean(o, fine, lf):
    """mean over the children of r/V, times the coarse volume"""
    Vf, Vc = o.volumes(lf), o.volumes(lf + 1)
    R = o.ratio(lf)
    q = fine / Vf
    nc = Vc.shape
    acc = np.zeros(nc)
    for a in range(R[0]):
        for b in range(R[1]):
            for c in range(R[2]):
                acc += q[a::R[0], b::R[1], c::R[2]][:nc[0], :nc[1], :nc[2]]
    return Vc * acc / (R[0] * R[1] * R[2])


def test_average_restriction_is_the_childrens_mean():
    o = Oracle(PTS, nthreads=2)
    o.assemble(restrict_average=1)
    rng = np.random.default_rng(1)
    for lf in range(o.num_levels - 1):
        fine = rng.standard_normal(o.shape(lf))
        assert np.allclose(o.restrict(lf, fine, scale=True), _children_mean(o, fine, lf), rtol=1e-14, atol=1e-14)
    # and it differs from the linear one on graded axes
    lin = Oracle(PTS, nthreads=2)
    lin.assemble()
    fine = rng.standard_normal(o.shape(0))
    assert not np.allclose(o.restrict(0, fine), lin.restrict(0, fine))


def test_injection_copies_the_parent():
    o = Oracle(PTS, nthreads=2)
    o.assemble(prolong_injection=1)
    rng = np.random.default_rng(2)
    for lf in range(o.num_levels - 1):
        R = o.ratio(lf)
        coarse = rng.standard_normal(o.shape(lf + 1))
        got = o.prolong(lf, coarse, np.zeros(o.shape(lf)), op="=")
        ref = np.repeat(np.repeat(np.repeat(coarse, R[0], 0), R[1], 1), R[2], 2)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("sweeps", [2, 3])
def test_pinned_coarse_smoothing_holds_the_first_cell(sweeps):
    """Smoothing the pinned coarse matrix (solver.C:201-231) keeps cell 0 at
    zero when its right-hand side is zero (MG.C:37-40): that matrix is the
    unpinned one with cell 0's row the identity and every coupling to cell 0
    removed, which is what the device's smoothers emulate by not updating
    cell 0."""
    o = Oracle(PTS, nthreads=2)
    o.assemble(coarse_level=1, coarse_direct=0)
    lc = o.num_levels - 2
    A = o.matrix(lc)
    assert A[0, 0, 0, 0] == 1.0 and np.all(A[0, 0, 0, 1:] == 0.0)
    # the neighbours of cell 0 no longer couple to it: slot 1 (lower x) of
    # cell (1,0,0), slot 3 (lower y) of (0,1,0), slot 5 (lower z) of (0,0,1)
    assert A[1, 0, 0, 1] == 0.0 and A[0, 1, 0, 3] == 0.0 and A[0, 0, 1, 5] == 0.0
    rng = np.random.default_rng(3)
    x = rng.standard_normal(o.shape(lc))
    b = rng.standard_normal(o.shape(lc))
    x.flat[0] = b.flat[0] = 0.0  # the cycle zeroes x and the pinned b (MG.C:37-45)
    got = o.smooth(lc, x, b, sweeps=sweeps)
    assert got.flat[0] == 0.0 and np.all(np.isfinite(got))
