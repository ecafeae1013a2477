"""CPU restatement of the reference's FFT Poisson solver -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU FFT solver; nothing in the
product imports it).

Follows, for one brick on one process:
  solve               src/briscolaFiniteVolume/solvers/PoissonSolvers/FFTPoissonSolver/FFTPoissonSolver.C:88-446
  transform kinds     .../FFTPoissonSolver/FourierTransforms/FourierTransforms.C:70-282 (boundary pair
                      codes, FFTW r2r kinds), :322-420 (normalisation)
  planner             .../FFTPoissonSolver/planner/planner.C:60-99 (solve direction: the first
                      non-uniform axis, else axis 0 when it has more than one cell)
  tridiagonal solve   .../FFTPoissonSolver/tridiagonalSolver/tridiagonalSolver.C:20-115 (eigenvalues),
                      :117-280 (diagonals, singular-mode pin), :330-374 (Thomas), :376-450 (cyclic)
  ghost cells         DirichletBoundaryCondition.C:51-71 (x_g = 2v - x_c),
                      NeumannBoundaryCondition.C:59-85 (x_g = x_c + g |c_c - c_g|)
  ghost points        src/briscolaMesh/level/levelPoints.C:198-236, 326-400
  known-answer check  applications/test/FFTPoissonSolver/Test-FFTPoissonSolver.C:11-92
  projection steps    divergenceScheme.C:116-150 (coloDiv of a staggered field),
                      exSchemesReconstruction.H:187-206 (stagReconstruct), briscolaStaggered.C:92-96
  split solver        src/briscolaFiniteVolume/solvers/PoissonSolvers/splitPoissonSolver/
                      splitPoissonSolver.C:53-155 (prediction, lambda0, modified source, corrections);
                      face gradient .../faceGradientSchemes/linearFaceGradientScheme/
                      linearFaceGradientScheme.C (outward through the lower face), flux divergence
                      .../divergenceSchemes/divergenceScheme/divergenceScheme.C:68-96

The FFTW r2r kinds are restated with scipy.fft, whose unnormalised DCT/DST
types 2, 3 and 4 have FFTW's REDFT10/01/11 and RODFT10/01/11 definitions;
R2HC/HC2R are numpy's real FFT in FFTW's halfcomplex order.  Parity of the
transforms is pinned by their definitions (tested against direct sums) and
of the whole solve by the reference's known-answer test.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

DIRICHLET, NEUMANN, PERIODIC, EMPTY = "Dirichlet", "Neumann", "periodic", "empty"

# FourierTransforms.C:130-226: boundary pair of an axis
PAIR_EMPTY, PAIR_DD, PAIR_NN, PAIR_DN, PAIR_ND, PAIR_CC = 0, 1, 2, 3, 4, 5


def pair_code(lo: str, hi: str) -> int:
    if lo == EMPTY:
        return PAIR_EMPTY
    if lo == PERIODIC:
        return PAIR_CC
    table = {(DIRICHLET, DIRICHLET): PAIR_DD, (NEUMANN, NEUMANN): PAIR_NN,
             (DIRICHLET, NEUMANN): PAIR_DN, (NEUMANN, DIRICHLET): PAIR_ND}
    if (lo, hi) not in table:
        raise ValueError(f"incorrect boundary condition pair {lo}-{hi}")
    return table[(lo, hi)]


def cell_sizes_with_ghosts(points: np.ndarray, periodic: bool) -> np.ndarray:
    """N+2 cell sizes, ghost cells included (levelPoints.C:198-236: a wall's
    ghost point mirrors the first spacing; :326-400: periodic ghosts take the
    opposite boundary spacing)."""
    h = np.diff(points)
    if periodic:
        return np.concatenate([[h[-1]], h, [h[0]]])
    return np.concatenate([[h[0]], h, [h[-1]]])


def is_uniform(points: np.ndarray, tol: float = 1e-12) -> bool:
    h = np.diff(points)
    return h.max() - h.min() <= tol


def solve_direction(points, n) -> int:
    """planner.C:60-99 on one process (decomposition type 0)."""
    for d in range(3):
        if not is_uniform(points[d]):
            return d
    return 0 if n[0] > 1 else 2


# ---- one-dimensional transforms (FourierTransforms.C:228-282) -------------

def r2hc(x: np.ndarray, axis: int) -> np.ndarray:
    """FFTW_R2HC: r_0..r_{N/2}, then i_{(N+1)/2-1}..i_1."""
    n = x.shape[axis]
    y = np.fft.rfft(x, axis=axis)
    out = np.empty_like(x)
    re = np.moveaxis(y.real, axis, -1)
    im = np.moveaxis(y.imag, axis, -1)
    o = np.moveaxis(out, axis, -1)
    half = n // 2
    o[..., :half + 1] = re[..., :half + 1]
    for k in range(1, (n + 1) // 2):
        o[..., n - k] = im[..., k]
    return out


def hc2r(x: np.ndarray, axis: int) -> np.ndarray:
    """FFTW_HC2R (unnormalised inverse of r2hc: hc2r(r2hc(x)) = N x)."""
    n = x.shape[axis]
    xi = np.moveaxis(x, axis, -1)
    spec = np.zeros(xi.shape[:-1] + (n // 2 + 1,), dtype=np.complex128)
    spec.real[..., :n // 2 + 1] = xi[..., :n // 2 + 1]
    for k in range(1, (n + 1) // 2):
        spec.imag[..., k] = xi[..., n - k]
    y = np.fft.irfft(spec, n=n, axis=-1) * n
    return np.moveaxis(y, -1, axis)


def forward(x: np.ndarray, axis: int, code: int) -> np.ndarray:
    """FourierTransforms.C:228-242: forward kinds RODFT10, REDFT10, RODFT11,
    REDFT11, R2HC for pairs D-D, N-N, D-N, N-D, C-C."""
    if code == PAIR_EMPTY:
        return x
    if code == PAIR_DD:
        return sfft.dst(x, type=2, axis=axis)
    if code == PAIR_NN:
        return sfft.dct(x, type=2, axis=axis)
    if code == PAIR_DN:
        return sfft.dst(x, type=4, axis=axis)
    if code == PAIR_ND:
        return sfft.dct(x, type=4, axis=axis)
    return r2hc(x, axis)


def backward(x: np.ndarray, axis: int, code: int) -> np.ndarray:
    """Backward kinds RODFT01, REDFT01, RODFT11, REDFT11, HC2R."""
    if code == PAIR_EMPTY:
        return x
    if code == PAIR_DD:
        return sfft.dst(x, type=3, axis=axis)
    if code == PAIR_NN:
        return sfft.dct(x, type=3, axis=axis)
    if code == PAIR_DN:
        return sfft.dst(x, type=4, axis=axis)
    if code == PAIR_ND:
        return sfft.dct(x, type=4, axis=axis)
    return hc2r(x, axis)


def normalisation(n: int, code: int) -> float:
    """FourierTransforms.C:322-420: N for C-C, 2N otherwise, 1 if empty."""
    if code == PAIR_EMPTY:
        return 1.0
    return float(n) if code == PAIR_CC else 2.0 * n


def eigenvalues(n: int, code: int) -> np.ndarray:
    """tridiagonalSolver.C:20-115, one process (Sd = 0)."""
    i = np.arange(n, dtype=np.float64)
    if code == PAIR_EMPTY:
        return np.zeros(n)
    if code == PAIR_DD:
        return -4.0 * np.sin((i + 1) * np.pi / (2.0 * n)) ** 2
    if code == PAIR_NN:
        return -4.0 * np.sin(i * np.pi / (2.0 * n)) ** 2
    if code in (PAIR_DN, PAIR_ND):
        return -4.0 * np.sin((2.0 * (i + 1) - 1.0) * np.pi / (4.0 * n)) ** 2
    return -4.0 * np.sin(i * np.pi / n) ** 2


# ---- tridiagonal solve (tridiagonalSolver.C:117-450) ----------------------

def transform_axes(s: int):
    """tridiagonalSolver.C:300-325: dir1, dir2 for each solve direction."""
    return {0: (2, 1), 1: (0, 2), 2: (0, 1)}[s]


def diagonals(h3g: np.ndarray, code: int, e: np.ndarray, singular: np.ndarray):
    """Main diagonal D (modes x Ns) and the couplings DU, DL (Ns) of
    tridiagonalSolver.C:117-280.  h3g: Ns+2 cell sizes with ghosts; e: the
    modes' eigenvalue sums; singular: modes whose eigenvalues are both 0."""
    ns = len(h3g) - 2
    d3 = h3g[1:-1]
    d3e = (h3g[1:-1] + h3g[2:]) / 2.0
    d3w = (h3g[1:-1] + h3g[:-2]) / 2.0
    D = e[:, None] - 1.0 / (d3e * d3)[None, :] - 1.0 / (d3 * d3w)[None, :]
    first_e = 1.0 / (d3e[0] * d3[0])
    first_w = 1.0 / (d3[0] * d3w[0])
    last_e = 1.0 / (d3e[-1] * d3[-1])
    last_w = 1.0 / (d3[-1] * d3w[-1])
    if code == PAIR_DD:
        D[:, 0] = e - first_e - 2.0 * first_w
        D[:, -1] = e - 2.0 * last_e - last_w
    elif code == PAIR_NN:
        D[:, 0] = e - first_e
        D[:, -1] = e - last_w
        D[singular, 0] = -first_e - 2.0 * first_w
    elif code == PAIR_DN:
        D[:, 0] = e - first_e - 2.0 * first_w
        D[:, -1] = e - last_w
    elif code == PAIR_ND:
        D[:, 0] = e - first_e
        D[:, -1] = e - 2.0 * last_e - last_w
    elif code == PAIR_CC:
        D[:, 0] = e - first_e - first_w
        D[:, -1] = e - last_e - last_w
        D[singular, 0] = -first_e - 2.0 * first_w
    else:
        raise ValueError("incorrect solve direction")
    DU = 1.0 / (d3 * d3e)
    DL = 1.0 / (d3 * d3w)
    return D, DU, DL


def thomas(D: np.ndarray, DU: np.ndarray, DL: np.ndarray, f: np.ndarray, start: int = 0) -> np.ndarray:
    """tridiagonalSolver.C:330-374 for every mode at once (rows of D, f)."""
    ns = D.shape[1]
    Dh = D.copy()
    fh = f.copy()
    for k in range(1 + start, ns):
        m = DL[k] / Dh[:, k - 1]
        Dh[:, k] -= m * DU[k - 1]
        fh[:, k] -= m * fh[:, k - 1]
    p = np.zeros_like(f)
    p[:, ns - 1] = fh[:, ns - 1] / Dh[:, ns - 1]
    for k in range(ns - 2, start - 1, -1):
        p[:, k] = (fh[:, k] - DU[k] * p[:, k + 1]) / Dh[:, k]
    return p


def thomas_cyclic(D, DU, DL, f):
    """tridiagonalSolver.C:376-450."""
    ns = D.shape[1]
    u = thomas(D, DU, DL, f, start=1)
    vf = np.zeros_like(f)
    vf[:, 1] = -DL[1]
    vf[:, ns - 1] = -DU[ns - 1]
    v = thomas(D, DU, DL, vf, start=1)
    p = np.empty_like(f)
    p[:, 0] = (f[:, 0] - DL[0] * u[:, ns - 1] - DU[0] * u[:, 1]) / (D[:, 0] + DL[0] * v[:, ns - 1] + DU[0] * v[:, 1])
    p[:, 1:] = u[:, 1:] + p[:, 0:1] * v[:, 1:]
    return p


# ---- the solve (FFTPoissonSolver.C:88-446) --------------------------------

def pairs(bc) -> list:
    return [pair_code(bc[2 * d], bc[2 * d + 1]) for d in range(3)]


def ghost_distance(points: np.ndarray, periodic: bool, side: int) -> float:
    """|c_c - c_g| across the lower (side 0) or upper (1) face."""
    h = cell_sizes_with_ghosts(points, periodic)
    return 0.5 * (h[0] + h[1]) if side == 0 else 0.5 * (h[-1] + h[-2])


def rhs(b: np.ndarray, points, bc, bc_values, shift: float = 0.0, x_old=None) -> np.ndarray:
    """FFTPoissonSolver.C:116-183: -b (minus x_old * shift for ddt), minus
    the inhomogeneous ghost contributions of Dirichlet and Neumann faces."""
    f = -np.asarray(b, dtype=np.float64).copy()
    if shift and x_old is not None:
        f -= shift * x_old
    n = f.shape
    for d in range(3):
        if bc[2 * d] in (PERIODIC, EMPTY):
            continue
        h = np.diff(points[d])
        for side in (0, 1):
            kind, val = bc[2 * d + side], bc_values[2 * d + side]
            if val == 0.0:
                continue
            idx = [slice(None)] * 3
            idx[d] = 0 if side == 0 else n[d] - 1
            hb = h[0] if side == 0 else h[-1]
            if kind == DIRICHLET:
                # (x_g + x_c) / h^2 with x_g = 2v - x_c
                f[tuple(idx)] -= 2.0 * val / hb ** 2
            else:
                # (x_g - x_c) / h^2 with x_g = x_c + g * dist
                f[tuple(idx)] -= val * ghost_distance(points[d], False, side) / hb ** 2
    return f


def solve(b: np.ndarray, points, bc, bc_values=(0.0,) * 6, shift: float = 0.0, x_old=None) -> np.ndarray:
    """x on the interior cells: Laplacian(x) - shift x = -b - shift x_old with
    the faces' Dirichlet values / Neumann gradients."""
    n = b.shape
    codes = pairs(bc)
    s = solve_direction(points, n)
    t1, t2 = transform_axes(s)
    f = rhs(b, points, bc, bc_values, shift, x_old)
    for a in (t1, t2):
        f = forward(f, a, codes[a])
    # modes: move the solve axis last
    perm = (t1, t2, s)
    g = np.transpose(f, perm)
    l1 = eigenvalues(n[t1], codes[t1])
    l2 = eigenvalues(n[t2], codes[t2])
    d1 = np.diff(points[t1])[0]
    d2 = np.diff(points[t2])[0]
    e = (l1[:, None] / d1 ** 2 + l2[None, :] / d2 ** 2).ravel()
    singular = ((l1[:, None] == 0) & (l2[None, :] == 0)).ravel()
    h3g = cell_sizes_with_ghosts(points[s], codes[s] == PAIR_CC)
    D, DU, DL = diagonals(h3g, codes[s], e, singular)
    D = D - shift
    G = g.reshape(-1, n[s])
    P = thomas_cyclic(D, DU, DL, G) if codes[s] == PAIR_CC else thomas(D, DU, DL, G)
    p = np.transpose(P.reshape(g.shape), np.argsort(perm))
    for a in (t2, t1):
        p = backward(p, a, codes[a])
    norm = normalisation(n[t1], codes[t1]) * normalisation(n[t2], codes[t2])
    return p / norm


# ---- the reference's known-answer check -----------------------------------

def with_ghosts(x: np.ndarray, points, bc, bc_values) -> np.ndarray:
    """x with a one-cell ghost frame set by the face conditions
    (correctBoundaryConditions: face ghosts only)."""
    n = x.shape
    g = np.zeros(tuple(m + 2 for m in n))
    g[1:-1, 1:-1, 1:-1] = x
    for d in range(3):
        lo = [slice(1, -1)] * 3
        hi = [slice(1, -1)] * 3
        c_lo = [slice(1, -1)] * 3
        c_hi = [slice(1, -1)] * 3
        lo[d], hi[d], c_lo[d], c_hi[d] = 0, n[d] + 1, 1, n[d]
        for side, gi, ci in ((0, lo, c_lo), (1, hi, c_hi)):
            kind, val = bc[2 * d + side], bc_values[2 * d + side]
            if kind in (PERIODIC, EMPTY):
                src = [slice(1, -1)] * 3
                src[d] = n[d] if side == 0 else 1
                g[tuple(gi)] = g[tuple(src)]
            elif kind == DIRICHLET:
                g[tuple(gi)] = 2.0 * val - g[tuple(ci)]
            else:
                g[tuple(gi)] = g[tuple(ci)] + val * ghost_distance(points[d], False, side)
    return g


def laplacian_residual(x: np.ndarray, f: np.ndarray, points, bc, bc_values) -> np.ndarray:
    """Test-FFTPoissonSolver.C:11-92: Laplacian(x) + f per cell, with face
    distances from the ghost-inclusive cell sizes."""
    g = with_ghosts(x, points, bc, bc_values)
    r = np.array(f, dtype=np.float64, copy=True)
    for d in range(3):
        h = cell_sizes_with_ghosts(points[d], bc[2 * d] == PERIODIC)
        hc = h[1:-1]
        dw = (h[1:-1] + h[:-2]) / 2.0
        de = (h[1:-1] + h[2:]) / 2.0
        shape = [1, 1, 1]
        shape[d] = -1
        hc, dw, de = (v.reshape(shape) for v in (hc, dw, de))
        c = [slice(1, -1)] * 3
        m = [slice(1, -1)] * 3
        p = [slice(1, -1)] * 3
        m[d] = slice(0, -2)
        p[d] = slice(2, None)
        xc, xm, xp = g[tuple(c)], g[tuple(m)], g[tuple(p)]
        r += xm / (dw * hc) - xc / (dw * hc) - xc / (de * hc) + xp / (de * hc)
    return r


# ---- split Poisson solver (splitPoissonSolver.C:53-155) --------------------

def face_flux_divergence(x, lamp, points, bc, bc_values):
    """div(lamp faceGrad(x) faceArea) per cell (volume-divided): faces of
    axis d carry lamp[d] ((n_d + 1) along d), ghosts from the face
    conditions (with_ghosts)."""
    g = with_ghosts(x, points, bc, bc_values)
    n = x.shape
    div = np.zeros(n)
    for d in range(3):
        if bc[2 * d] == EMPTY:
            continue
        h = cell_sizes_with_ghosts(points[d], bc[2 * d] == PERIODIC)
        delta = 1.0 / ((h[1:] + h[:-1]) / 2.0)  # n+1 faces: between ghost/interior cells
        shape = [1, 1, 1]
        shape[d] = -1
        delta = delta.reshape(shape)
        # outward gradient through the lower face of cell q (q = 0..n): x[q-1] - x[q]
        lo = [slice(1, -1)] * 3
        hi = [slice(1, -1)] * 3
        lo[d] = slice(0, n[d] + 1)
        hi[d] = slice(1, n[d] + 2)
        grad = (g[tuple(lo)] - g[tuple(hi)]) * delta
        phi = lamp[d] * grad
        # Div(cell q) += phi(face q); Div(cell q-1) -= phi(face q)
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[d] = slice(0, n[d])
        b[d] = slice(1, n[d] + 1)
        hc = np.diff(points[d]).reshape(shape)
        div += (phi[tuple(a)] - phi[tuple(b)]) / hc
    return div


def split_source(x, b, lam, lambda0, points, bc, bc_values=(0.0,) * 6):
    """bhat = b / lambda0 + div((lambda / lambda0 - 1) faceGrad(x) faceArea)
    (splitPoissonSolver.C:118-138)."""
    lamp = [l / lambda0 - 1.0 for l in lam]
    return b / lambda0 + face_flux_divergence(x, lamp, points, bc, bc_values)


def split_solve(x, b, lam, points, bc, bc_values=(0.0,) * 6, n_corr=1):
    """nCorr corrections of the split solver from the initial x (prediction
    and preconditioner applied by the caller), FFT inner solver."""
    lambda0 = max(float(l.max()) for l in lam)
    for _ in range(n_corr):
        bhat = split_source(x, b, lam, lambda0, points, bc, bc_values)
        x = solve(bhat, points, bc, bc_values)
    return x


def variable_residual(x, b, lam, points, bc, bc_values=(0.0,) * 6):
    """-div(lambda grad x) - b per cell: the equation the split solver
    approximates."""
    return -face_flux_divergence(x, lam, points, bc, bc_values) - b


# ---- projection steps either side of the pressure solve -------------------

def colo_div(u, points):
    """coloDiv of a staggered field (divergenceScheme.C:116-150): the face
    arrays u[d] hold n_d + 1 faces along d; sum of U A over the faces / V."""
    n = tuple(len(p) - 1 for p in points)
    div = np.zeros(n)
    for d in range(3):
        shape = [1, 1, 1]
        shape[d] = -1
        hc = np.diff(points[d]).reshape(shape)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[d] = slice(0, n[d])
        hi[d] = slice(1, n[d] + 1)
        div += (u[d][tuple(hi)] - u[d][tuple(lo)]) / hc
    return div


def project_correct(u, p, c_dt, points, periodic, lam=None):
    """U - c_dt stagReconstruct(lambda faceGrad(p) A) (briscolaStaggered.C:96,
    exSchemesReconstruction.H:187-206): face q of axis d loses
    c_dt lambda (p_q - p_{q-1}) delta; walls keep their faces (zero
    gradient), periodic faces wrap."""
    out = [a.copy() for a in u]
    n = p.shape
    for d in range(3):
        h = cell_sizes_with_ghosts(points[d], periodic[d])
        delta = 1.0 / ((h[1:] + h[:-1]) / 2.0)  # faces 0..n
        shape = [1, 1, 1]
        shape[d] = -1
        ext = np.concatenate([np.take(p, [n[d] - 1], axis=d), p, np.take(p, [0], axis=d)], axis=d)
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[d] = slice(1, n[d] + 2)
        b[d] = slice(0, n[d] + 1)
        g = (ext[tuple(a)] - ext[tuple(b)]) * delta.reshape(shape)
        if not periodic[d]:
            first = [slice(None)] * 3
            last = [slice(None)] * 3
            first[d], last[d] = 0, n[d]
            g[tuple(first)] = 0.0
            g[tuple(last)] = 0.0
        lf = 1.0 if lam is None else lam[d]
        out[d] = out[d] - c_dt * (lf * g)
    return out
