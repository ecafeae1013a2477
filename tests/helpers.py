"""Shared test helpers: independent FP64 ground truths and mesh builders."""
from __future__ import annotations

import numpy as np
from scipy.fft import dctn, idctn


def uniform(n, L=1.0):
    return L * np.arange(n + 1, dtype=np.float64) / n


def dct_neumann_solution(b: np.ndarray, h: float) -> np.ndarray:
    """Solve A x = b for the uniform cell-centred all-Neumann Laplacian of the
    reference (face coefficient area*delta = h on a cube of spacing h) by
    DCT-II diagonalisation; the null-space component is dropped."""
    n0, n1, n2 = b.shape
    lam = [2.0 * np.cos(np.pi * np.arange(n) / n) - 2.0 for n in (n0, n1, n2)]
    L = h * (lam[0][:, None, None] + lam[1][None, :, None] + lam[2][None, None, :])
    bh = dctn(b, type=2, norm="ortho")
    L[0, 0, 0] = 1.0
    xh = bh / L
    xh[0, 0, 0] = 0.0
    return idctn(xh, type=2, norm="ortho")


def channel_solution(b: np.ndarray, px, py, pz) -> np.ndarray:
    """FFT in the periodic x and z directions, tridiagonal (Thomas) solve in
    the walled y direction -- the method of the reference's FFT Poisson
    solver.  b is the unscaled system RHS; x and z uniform."""
    n0, n1, n2 = b.shape
    hx = px[1] - px[0]
    hz = pz[1] - pz[0]
    hy = np.diff(py)
    yc = 0.5 * (py[1:] + py[:-1])
    dy = np.diff(yc)  # centre distances of interior y faces
    # divide by the cell volume: (1/V) A x = b/V
    bs = b / (hx * hy[None, :, None] * hz)
    bh = np.fft.fft2(bs, axes=(0, 2))
    kx = np.fft.fftfreq(n0) * n0
    kz = np.fft.fftfreq(n2) * n2
    ex = (2 * np.cos(2 * np.pi * kx / n0) - 2) / hx**2
    ez = (2 * np.cos(2 * np.pi * kz / n2) - 2) / hz**2
    lo = np.zeros(n1)
    up = np.zeros(n1)
    lo[1:] = 1.0 / (dy * hy[1:])
    up[:-1] = 1.0 / (dy * hy[:-1])
    xh = np.zeros_like(bh)
    for a in range(n0):
        for c in range(n2):
            diag = -(lo + up) + ex[a] + ez[c]
            rhs = bh[a, :, c].copy()
            if a == 0 and c == 0:
                # singular mode: pin the first unknown
                d = diag.copy()
                u = up.copy()
                l_ = lo.copy()
                d[0] = 1.0
                u[0] = 0.0
                l_[1] = 0.0
                rhs[0] = 0.0
                xh[a, :, c] = thomas(l_, d, u, rhs)
            else:
                xh[a, :, c] = thomas(lo, diag, up, rhs)
    return np.real(np.fft.ifft2(xh, axes=(0, 2)))


def thomas(lo, d, up, r):
    n = len(d)
    c = np.zeros(n, dtype=complex)
    g = np.zeros(n, dtype=complex)
    c[0] = up[0] / d[0]
    g[0] = r[0] / d[0]
    for i in range(1, n):
        m = d[i] - lo[i] * c[i - 1]
        c[i] = up[i] / m if i < n - 1 else 0.0
        g[i] = (r[i] - lo[i] * g[i - 1]) / m
    x = np.zeros(n, dtype=complex)
    x[-1] = g[-1]
    for i in range(n - 2, -1, -1):
        x[i] = g[i] - c[i] * x[i + 1]
    return x


def vmean(x, V):
    return x - (V * x).sum() / V.sum()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
