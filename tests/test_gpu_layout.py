"""Parity-split rows (rowLayout split, the default) against natural rows.

On single-brick levels above 4096 cells with n2 % 16 == 0 the device keeps
each row's even-k cells first, then its odd-k cells; the per-cell
arithmetic of every kernel is unchanged, so solves with either layout must
agree bit for bit, whatever the precision, cycle, smoother, coefficient or
wall condition.  The one exception is the flexible-CG outer loop: on a
split level 0 its direction kernel adds its per-block partial sums over
cells of one parity, so the inner products round differently and the
solutions agree to the solve's accuracy (relative 1e-9 at relTol 1e-10)
with the same cycle count.  The building blocks on split levels are also
checked against the CPU oracle, as the natural ones are in
test_gpu_parity.py.
"""
import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import workloads
from briscola_b200.mesh import NEUMANN, PERIODIC, Brick, Mesh, geometric_points, tanh_points, uniform_points
from oracle.pyoracle import Oracle
from tests.helpers import rel

pytestmark = pytest.mark.gpu

V22 = {"nSweepsPre": 2, "nSweepsPost": 2, "cycleType": "V", "coarseLevel": 1, "tolerance": 0}


def _solve(mesh, b, layout, lam=None, **kw):
    d = dict(V22)
    d.update(kw)
    d["rowLayout"] = layout
    c = bb.Context(mesh, bb.make_options(d))
    if lam is not None:
        c.set_coefficients(lam)
    x = np.zeros_like(b)
    rep = c.solve(b, x, zero_guess=True)
    x2 = np.zeros_like(b)
    rep2 = c.solve(b, x2, zero_guess=True)  # the replayed graph gives the same
    c.close()
    assert np.array_equal(x, x2)
    return x, rep


def _graded_k(N):
    br = Brick([uniform_points(N), geometric_points(N, 2.0), geometric_points(N, 0.5)], (NEUMANN,) * 6)
    rng = np.random.default_rng(9)
    V = br.cell_volumes()
    f = rng.standard_normal(br.N)
    f -= (V * f).sum() / V.sum()
    return Mesh([br]), np.ascontiguousarray((-V * f).ravel()), None


def _dirichlet(N):
    br = Brick([uniform_points(N), tanh_points(N, 2.0), uniform_points(N)],
               ("Dirichlet", "Neumann", "periodic", "periodic", "Dirichlet", "Dirichlet"),
               values=(1.0, 0.5, 0.0, 0.0, -2.0, 0.25))
    rng = np.random.default_rng(4)
    return Mesh([br]), rng.standard_normal(N ** 3), None


def _thin_rows(N=32):
    """rows of 16 cells, the narrowest split rows: two threads a half row in
    FP32, four in FP64; periodic x and z, stretched walls in y"""
    br = Brick([uniform_points(N), geometric_points(N, 2.0), uniform_points(16)],
               (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC))
    rng = np.random.default_rng(12)
    V = br.cell_volumes()
    f = rng.standard_normal(br.N)
    f -= (V * f).sum() / V.sum()
    return Mesh([br]), np.ascontiguousarray((-V * f).ravel()), None


CASES = {
    "channel_fp64": (lambda: workloads.channel(64), dict(relTol=1e-10, precision="fp64")),
    "channel_mixed_fcg": (lambda: workloads.channel(64), dict(relTol=1e-10, precision="mixed", krylov="fcg")),
    "channel_mixed": (lambda: workloads.channel(64), dict(relTol=1e-9, precision="mixed")),
    "cavity_fp64_fcg": (lambda: workloads.cavity(64), dict(relTol=1e-10, precision="fp64", krylov="fcg")),
    "sphere_fp64": (lambda: workloads.sphere(64), dict(relTol=1e-9, precision="fp64", maxIter=200)),
    "sphere_mixed_fcg": (lambda: workloads.sphere(64),
                         dict(relTol=1e-9, precision="mixed", krylov="fcg", maxIter=200)),
    "graded_k_fp64": (lambda: _graded_k(48), dict(relTol=1e-10, precision="fp64")),
    "dirichlet_fp64": (lambda: _dirichlet(64), dict(relTol=1e-10, precision="fp64")),
    "dirichlet_mixed_fcg": (lambda: _dirichlet(64), dict(relTol=1e-10, precision="mixed", krylov="fcg")),
    "w_cycle": (lambda: workloads.channel(64), dict(relTol=1e-10, cycleType="W")),
    "f_cycle_mixed": (lambda: workloads.channel(64), dict(relTol=1e-9, cycleType="F", precision="mixed")),
    "jacobi": (lambda: workloads.channel(64), dict(relTol=1e-9, smoother="jac", maxIter=300)),
    "no_coarse_fusion": (lambda: workloads.channel(64), dict(relTol=1e-10, fuseCoarse="off")),
    # twelve cycles whose smoothed coarse level (32^3) is split and pinned
    "coarse_smooth": (lambda: workloads.cavity(64), dict(relTol=1e-14, coarseMode="smooth", coarseLevel=3,
                                                         maxIter=12)),
    "no_graph": (lambda: workloads.channel(64), dict(relTol=1e-10, graph="off", precision="mixed",
                                                     krylov="fcg")),
    "thin_rows_fp64": (_thin_rows, dict(relTol=1e-10, precision="fp64")),
    "thin_rows_mixed": (_thin_rows, dict(relTol=1e-9, precision="mixed")),
    "thin_rows_mixed_fcg": (_thin_rows, dict(relTol=1e-10, precision="mixed", krylov="fcg")),
}


@pytest.mark.parametrize("name", list(CASES))
def test_split_rows_are_bit_identical_to_natural(native, name):
    make, kw = CASES[name]
    mesh, b, lam = make()
    xs, rs = _solve(mesh, b, "split", lam, **kw)
    xn, rn = _solve(mesh, b, "natural", lam, **kw)
    assert rs.status == rn.status and rs.cycles == rn.cycles
    assert rs.status == 0 or name == "coarse_smooth", rs.status
    if kw.get("krylov") == "fcg":
        assert rel(xs - xs.mean(), xn - xn.mean()) <= 1e-9
    else:
        assert np.array_equal(xs, xn), float(np.abs(xs - xn).max())


def test_split_levels_are_in_use(native):
    """The 64^3 channel's two finest levels are split (the bit-identity test
    above would pass vacuously otherwise): their colour passes take a
    different kernel, so the launch counts agree but the layout differs in
    memory -- the level arrays read back through the C ABI are unchanged."""
    mesh, b, _ = workloads.channel(64)
    c = bb.Context(mesh, bb.make_options(dict(V22, rowLayout="split")))
    rng = np.random.default_rng(2)
    x = rng.standard_normal(c.shape(0))
    c.upload(0, "x", x)
    assert np.array_equal(c.download(0, "x"), x)
    c.close()


def _oracle(br, lam=None):
    o = Oracle(br.points, periodic=br.periodic, nthreads=4)
    if lam is not None:
        o.set_lambda(*lam)
    o.assemble(n_pre=2, n_post=2, cycle_type="V", coarse_level=1)
    return o


SPLIT_MESHES = {
    "walls_graded_k": lambda: Brick([uniform_points(16), geometric_points(16, 2.0), geometric_points(32, 0.5)]),
    "channel": lambda: Brick([uniform_points(32), tanh_points(16, 2.0), uniform_points(64)],
                             (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC)),
    "all_periodic": lambda: Brick([uniform_points(16), uniform_points(16), uniform_points(32)], (PERIODIC,) * 6),
}


def _lam(br, seed):
    rng = np.random.default_rng(seed)
    n0, n1, n2 = br.N
    lam = [np.exp(rng.uniform(-2, 2, s)) for s in ((n0 + 1, n1, n2), (n0, n1 + 1, n2), (n0, n1, n2 + 1))]
    for d in range(3):  # a periodic face is one face: both copies equal
        if br.periodic[d]:
            sl0 = [slice(None)] * 3
            sl1 = [slice(None)] * 3
            sl0[d], sl1[d] = 0, -1
            lam[d][tuple(sl1)] = lam[d][tuple(sl0)]
    return lam


@pytest.mark.parametrize("name", list(SPLIT_MESHES))
@pytest.mark.parametrize("variable", [False, True])
@pytest.mark.parametrize("precision", [0, 1])
def test_split_level_kernels_match_oracle(native, name, variable, precision):
    """Level 0 of these bricks is split (above 4096 cells, n2 % 16 == 0):
    colour passes, residual, restriction into the (natural) next level and
    prolongation from it, against the oracle (FP64 1e-13, FP32 2e-6)."""
    br = SPLIT_MESHES[name]()
    lam = _lam(br, 3) if variable else None
    c = bb.Context(Mesh([br]), bb.make_options(dict(V22)))
    if lam is not None:
        c.set_coefficients(lam)
    o = _oracle(br, lam)
    tol = 1e-13 if precision == 0 else 2e-6
    rng = np.random.default_rng(5)
    shp = c.shape(0)
    x = rng.standard_normal(shp)
    b = rng.standard_normal(shp)
    c.upload(0, "b", b, precision=precision)
    for colour in (0, 1):
        c.upload(0, "x", x, precision=precision)
        c.colour_pass(0, colour, precision=precision)
        assert rel(c.download(0, "x", precision=precision), o.colour_pass(0, colour, x, b)) <= tol, colour
    c.upload(0, "x", x, precision=precision)
    r_ref = o.residual(0, x, b)
    if precision == 0:
        assert rel(c.residual(0), r_ref) <= tol
    c.residual_restrict(0, precision=precision)
    assert rel(c.download(1, "b", precision=precision), o.restrict(0, r_ref, scale=True)) <= tol
    xc = rng.standard_normal(c.shape(1))
    c.upload(1, "x", xc, precision=precision)
    c.upload(0, "x", x, precision=precision)
    c.prolong_correct(0, precision=precision)
    assert rel(c.download(0, "x", precision=precision), o.prolong(0, xc, x, op="+=")) <= tol
    c.close()


@pytest.mark.parametrize("case", ["channel", "cavity"])
def test_first_pass_fusion_is_bit_identical(native, case):
    """With fuseFirstPass on (the default) each FP32 cycle of the flexible-CG
    loop starts with a zero-start colour pass on the split level 0, which
    reads no z and writes the whole level; the solve is bit-identical to the
    one that zeroes z with a memset and runs the ordinary pass."""
    mesh, b, _ = workloads.CONFIGS[case](64)
    kw = dict(relTol=1e-10, precision="mixed", krylov="fcg")
    out = {}
    for f in ("on", "off"):
        d = dict(V22, fuseFirstPass=f, **kw)
        c = bb.Context(mesh, bb.make_options(d))
        x = np.zeros_like(b)
        rep = c.solve(b, x, zero_guess=True)
        assert rep.status == 0
        out[f] = (x, rep.cycles, rep.kernel_launches)
        c.close()
    assert out["on"][1] == out["off"][1] and np.array_equal(out["on"][0], out["off"][0])
    assert out["on"][2] == out["off"][2]  # the same kernels; the memset is gone
