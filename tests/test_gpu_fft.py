"""The B200 FFT Poisson solver (csrc/bfft.cu through include/bfft.h) against
the CPU restatement of the reference's FFT solver (oracle/fft_oracle.py):
the reference's known-answer tests (mixed Dirichlet / Neumann faces with
values, each direction stretched in turn; the ddt form), periodic and
singular configurations, device-pointer solves on torch's stream, and the
256^3 channel.  FP64 throughout: solutions agree to 1e-12 relative and the
discrete Laplacian residual stays within the reference's 1e-10."""
import numpy as np
import pytest

from briscola_b200 import fft
from briscola_b200.mesh import DIRICHLET, EMPTY, NEUMANN, PERIODIC, Brick, geometric_points, tanh_points, uniform_points
from oracle import fft_oracle as F

pytestmark = pytest.mark.gpu

D, N, P = DIRICHLET, NEUMANN, PERIODIC
REF_BC = (D, D, N, N, N, D)
REF_VALUES = (1.0, 2.0, 3.0, 4.0, 5.0, 6.0)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("stretch", [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2)])
def test_known_answer_mixed_faces(stretch):
    n = (16, 64, 32)
    pts = [geometric_points(n[d], stretch[d]) for d in range(3)]
    rng = np.random.default_rng(123)
    f = 100.0 * rng.random(n) - 0.5
    f -= f.mean()
    s = fft.FFTPoissonSolver(Brick(pts, REF_BC), REF_VALUES)
    x = s.solve(None, f)
    ref = F.solve(f, pts, REF_BC, REF_VALUES)
    assert s.solve_direction == F.solve_direction(pts, n)
    assert rel(x, ref) <= 1e-12
    r = F.laplacian_residual(x, f, pts, REF_BC, REF_VALUES)
    assert np.abs(r).max() <= 1e-10 * max(1.0, np.abs(f).max() / 100.0)


@pytest.mark.parametrize("bc,stretch_axis", [
    ((P, P, N, N, P, P), 1),   # channel
    ((N, N, N, N, N, N), 0),   # closed box, pinned mean mode
    ((P, P, P, P, P, P), None),  # triply periodic: cyclic tridiagonal
    ((D, N, P, P, N, D), 0),
    ((N, D, D, N, P, P), None),  # uniform: N-D solve along x, D-N and periodic transforms
    # zero-eigenvalue modes of the transforms that are not singular (a
    # Dirichlet face in the solve direction): no pin
    ((P, P, D, D, P, P), 1),     # channel with Dirichlet walls
    ((N, N, D, N, N, N), 1),     # closed box with one Dirichlet wall, D-N solve
])
def test_configurations_match_oracle(bc, stretch_axis):
    n = [16, 32, 8]
    pts = [uniform_points(m) for m in n]
    if stretch_axis is not None and bc[2 * stretch_axis] != P:
        pts[stretch_axis] = geometric_points(n[stretch_axis], 3.0)
    rng = np.random.default_rng(11)
    f = rng.standard_normal(tuple(n))
    if all(c in (N, P) for c in bc):
        V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
        f -= (f * V).sum() / V.sum()
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    x = s.solve(None, f)
    ref = F.solve(f, pts, bc)
    assert rel(x, ref) <= 1e-12
    assert np.abs(F.laplacian_residual(x, f, pts, bc, (0.0,) * 6)).max() <= 1e-9


@pytest.mark.parametrize("bc,n", [
    ((P, P, EMPTY, EMPTY, N, N), (16, 1, 32)),  # two-dimensional: an empty axis
    ((N, N, P, P, D, D), (16, 1, 8)),           # a periodic axis of one cell
    ((D, D, N, D, N, N), (8, 4, 7)),            # stretched z of 7 cells: odd k rows, single-element copies
])
def test_thin_and_ragged_shapes(bc, n):
    pts = [uniform_points(m) for m in n]
    if n[2] == 7:
        pts[2] = geometric_points(7, 2.0)
    rng = np.random.default_rng(13)
    f = rng.standard_normal(n)
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    x = s.solve(None, f)
    ref = F.solve(f, pts, bc)
    assert rel(x, ref) <= 1e-12


@pytest.mark.parametrize("bc,n", [
    ((D, D, N, N, P, P), (2, 16, 4)),  # sine pair of two lines, periodic of four
    ((N, N, D, D, N, N), (4, 8, 2)),   # cosine transforms of four and two points
    ((P, P, N, N, D, D), (2, 8, 2)),   # real FFT and sine of two points
    ((N, N, N, N, D, D), (1, 8, 4)),   # a cosine transform of one point
    ((D, D, N, N, N, N), (1, 8, 2)),   # a sine transform of one point
])
def test_tiny_transform_extents(bc, n):
    """Transform axes of 1, 2 and 4 cells: the paired real FFTs and
    Makhoul's cosine and sine transforms at their smallest lengths (no or
    one Stockham pass), against the restatement; y is stretched, so it is
    the solve direction."""
    pts = [uniform_points(m) for m in n]
    pts[1] = geometric_points(n[1], 2.0)
    rng = np.random.default_rng(17)
    f = rng.standard_normal(n)
    if all(c in (N, P) for c in bc):
        V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
        f -= (f * V).sum() / V.sum()
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    x = s.solve(None, f)
    ref = F.solve(f, pts, bc)
    assert rel(x, ref) <= 1e-12


def test_known_answer_ddt():
    n = (16, 16, 16)
    pts = [uniform_points(m) for m in n]
    bc = (D,) * 6
    rng = np.random.default_rng(7)
    b = rng.random(n) - 0.5
    xo = rng.random(n) - 0.5
    dt = 0.01
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    x = s.solve(None, b, ddt=True, dt=dt, x_old=xo)
    ref = F.solve(b, pts, bc, shift=1.0 / dt, x_old=xo)
    assert rel(x, ref) <= 1e-12
    r = F.laplacian_residual(x, b + xo / dt, pts, bc, (0.0,) * 6) - x / dt
    assert np.abs(r).max() <= 1e-10 / dt


def test_device_pointers_follow_torch_stream():
    torch = pytest.importorskip("torch")
    n = (32, 64, 32)
    pts = [uniform_points(32), tanh_points(64, 2.0), uniform_points(32)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(n)
    f -= f.mean()
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        torch.cuda._sleep(20_000_000)  # the solve must wait for this copy, not race it
        b = torch.from_numpy(f).cuda(non_blocking=False)
        x = torch.empty_like(b)
        s.solve(x, b)
        out = x.cpu().numpy()
    ref = F.solve(f, pts, bc)
    assert rel(out, ref) <= 1e-12


def test_refuses_what_the_reference_refuses():
    pts = [uniform_points(16), uniform_points(16), uniform_points(16)]
    with pytest.raises(fft.FatalError):
        fft.FFTPoissonSolver(Brick([pts[0], geometric_points(16, 2.0), geometric_points(16, 2.0)], (N,) * 6))
    s = fft.FFTPoissonSolver(Brick(pts, (N,) * 6))
    with pytest.raises(fft.FatalError):
        s.solve(None, np.zeros((16, 16, 16)), lam=np.ones(3))
    with pytest.raises(fft.FatalError):  # a transformed extent that is not a power of two
        fft.FFTPoissonSolver(Brick([uniform_points(16), uniform_points(12), uniform_points(16)], (N,) * 6))


def test_channel_256():
    n = (256, 256, 256)
    pts = [uniform_points(256, 2 * np.pi), tanh_points(256, 2.0), uniform_points(256, np.pi)]
    bc = (P, P, N, N, P, P)
    rng = np.random.default_rng(0)
    f = rng.standard_normal(n)
    V = np.diff(pts[0])[:, None, None] * np.diff(pts[1])[None, :, None] * np.diff(pts[2])[None, None, :]
    f -= (f * V).sum() / V.sum()
    s = fft.FFTPoissonSolver(Brick(pts, bc))
    x = s.solve(None, f)
    ref = F.solve(f, pts, bc)
    assert rel(x, ref) <= 1e-11
    r = F.laplacian_residual(x, f, pts, bc, (0.0,) * 6)
    assert np.abs(r).max() <= 1e-10 * max(1.0, np.abs(f).max())
