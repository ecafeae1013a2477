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


# ---------------------------------------------------------------------------
# multi-brick meshes: the union-domain operator as an independent ground truth
# ---------------------------------------------------------------------------
def split_brick(brick, cuts):
    """Split one brick into the product of the pieces between cut indices
    (cuts[d] lists interior cell indices along axis d).  The pieces take
    slices of the same coordinate arrays, so the union is the same mesh."""
    from briscola_b200.mesh import Brick, Mesh

    edges = [[0] + sorted(cuts[d]) + [brick.N[d]] for d in range(3)]
    bricks = []
    for a in range(len(edges[0]) - 1):
        for b in range(len(edges[1]) - 1):
            for c in range(len(edges[2]) - 1):
                lo = (edges[0][a], edges[1][b], edges[2][c])
                hi = (edges[0][a + 1], edges[1][b + 1], edges[2][c + 1])
                pts = [brick.points[d][lo[d]:hi[d] + 1] for d in range(3)]
                bricks.append(Brick(pts, brick.bc, lo, brick.values))
    return Mesh(bricks)


def brick_to_compact(mesh, full):
    """A field on the split brick's full (n0, n1, n2) array -> the C ABI's
    order for the pieces (bricks one after another, k fastest)."""
    parts = []
    for br in mesh.bricks:
        o, n = br.origin, br.N
        parts.append(full[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]].ravel())
    return np.concatenate(parts)


def union_operator(mesh):
    """Sparse FV Laplacian on the union of the bricks' cells: off-diagonal =
    face area / centre distance (linearGaussLaplacianScheme.C:59-94 with
    delta = 1/|cc_P - cc_N|), centre = -(sum of the row), Neumann outer walls.
    Rows in the C ABI's order.  Returns (A, V) with V the cell volumes."""
    import scipy.sparse as sp

    lo = np.min([br.origin for br in mesh.bricks], axis=0)
    hi = np.max([np.add(br.origin, br.N) for br in mesh.bricks], axis=0)
    index = -np.ones(tuple(hi - lo), dtype=np.int64)
    cc = [[], [], []]
    hh = [[], [], []]
    row0 = 0
    for br in mesh.bricks:
        n = br.N
        o = np.subtract(br.origin, lo)
        index[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]] = row0 + np.arange(np.prod(n)).reshape(n)
        grids = np.meshgrid(*[br.cell_centres(d) for d in range(3)], indexing="ij")
        sizes = np.meshgrid(*[br.cell_sizes(d) for d in range(3)], indexing="ij")
        for d in range(3):
            cc[d].append(grids[d].ravel())
            hh[d].append(sizes[d].ravel())
        row0 += int(np.prod(n))
    cc = [np.concatenate(a) for a in cc]
    hh = [np.concatenate(a) for a in hh]
    rows, cols, vals = [], [], []
    for d in range(3):
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[d] = slice(0, -1)
        sl_b[d] = slice(1, None)
        p = index[tuple(sl_a)].ravel()
        q = index[tuple(sl_b)].ravel()
        ok = (p >= 0) & (q >= 0)
        p, q = p[ok], q[ok]
        t1, t2 = (d + 1) % 3, (d + 2) % 3
        w = hh[t1][p] * hh[t2][p] / np.abs(cc[d][q] - cc[d][p])
        rows += [p, q]
        cols += [q, p]
        vals += [w, w]
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    n = row0
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A = A - sp.diags(np.asarray(A.sum(axis=1)).ravel())
    V = hh[0] * hh[1] * hh[2]
    return A.tocsr(), V


def union_operator_bc(mesh):
    """union_operator with each brick's own conditions on its wall faces
    (faces, or the cells of a face, with no brick beyond them; the mesh has
    no periodic axis): a Dirichlet wall adds its coefficient area / h once
    more to the centre and moves -2 (area / h) g to the right-hand side, a
    Neumann wall with gradient g moves -area g there (the rules of
    brick_operator, DirichletBoundaryCondition.C:19-51,
    NeumannBoundaryCondition.C:19-56).  Returns (A, V, bdir)."""
    import scipy.sparse as sp

    A, V = union_operator(mesh)
    lo = np.min([br.origin for br in mesh.bricks], axis=0)
    hi = np.max([np.add(br.origin, br.N) for br in mesh.bricks], axis=0)
    occupied = np.zeros(tuple(hi - lo), dtype=bool)
    for br in mesh.bricks:
        o = np.subtract(br.origin, lo)
        occupied[o[0]:o[0] + br.N[0], o[1]:o[1] + br.N[1], o[2]:o[2] + br.N[2]] = True
    ntot = A.shape[0]
    diag = np.zeros(ntot)
    bdir = np.zeros(ntot)
    row0 = 0
    for br in mesh.bricks:
        n = br.N
        idx = row0 + np.arange(int(np.prod(n))).reshape(n)
        h = [br.cell_sizes(d) for d in range(3)]
        o = np.subtract(br.origin, lo)
        for d in range(3):
            t1, t2 = (d + 1) % 3, (d + 2) % 3
            for side in range(2):
                kind, g = br.bc[2 * d + side], br.values[2 * d + side]
                cell = 0 if side == 0 else n[d] - 1
                outside = o[d] - 1 if side == 0 else o[d] + n[d]
                sl = [slice(None)] * 3
                sl[d] = slice(cell, cell + 1)
                C = np.squeeze(idx[tuple(sl)], axis=d)  # (n[a], n[b]), a < b the two tangential axes
                ta, tb = sorted((t1, t2))
                area = h[ta][:, None] * h[tb][None, :]
                if 0 <= outside < occupied.shape[d]:
                    osl = [slice(None)] * 3
                    osl[d] = outside
                    osl[ta] = slice(o[ta], o[ta] + n[ta])
                    osl[tb] = slice(o[tb], o[tb] + n[tb])
                    wall = ~occupied[tuple(osl)]
                else:
                    wall = np.ones((n[ta], n[tb]), dtype=bool)
                if kind == "Dirichlet":
                    a = area / h[d][cell]
                    diag[C[wall]] -= 2.0 * a[wall]
                    bdir[C[wall]] -= 2.0 * a[wall] * g
                elif kind == "Neumann" and g != 0.0:
                    bdir[C[wall]] -= area[wall] * g
        row0 += int(np.prod(n))
    return (A + sp.diags(diag)).tocsr(), V, bdir


def union_solve(mesh, b):
    """Direct FP64 solve of the union-domain Neumann problem with the
    reference's pin (first unknown fixed, solver.C:201-231), then the
    volume-weighted mean removed."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    A, V = union_operator(mesh)
    A = A.tolil()
    A[0, :] = 0.0
    A[:, 0] = 0.0
    A[0, 0] = 1.0
    rhs = b.copy()
    rhs[0] = 0.0
    x = spl.spsolve(sp.csc_matrix(A), rhs)
    return vmean(x, V), V


def brick_operator(points, bc, values=(0.0,) * 6, lam=None):
    """Sparse FV Laplacian of one brick with periodic, Neumann and Dirichlet
    faces, written from the reference's rules independently of the oracle:
    off-diagonal area * delta * lambda (delta = 1/|cc_P - cc_N|, a wall's
    ghost centre one first spacing beyond the wall, levelPoints.C:198-236),
    centre minus the row; a Neumann wall drops its face and moves
    -A_f g / delta to the right-hand side (gradient g,
    NeumannBoundaryCondition.C:19-56), a Dirichlet wall adds its coefficient
    once more to the centre and moves -2 A_f g there (value g,
    DirichletBoundaryCondition.C:19-51).  bc: "periodic",
    "Neumann" or "Dirichlet" per face (x-lo, x-hi, y-lo, ...).  Returns
    (A, V, bdir): rows k fastest, V the cell volumes, bdir the right-hand-side
    term of the Dirichlet values (add it to b_sys)."""
    import scipy.sparse as sp

    pts = [np.asarray(p, dtype=np.float64) for p in points]
    n = tuple(len(p) - 1 for p in pts)
    ntot = int(np.prod(n))
    idx = np.arange(ntot).reshape(n)
    h = [np.diff(p) for p in pts]
    cc = [0.5 * (p[1:] + p[:-1]) for p in pts]
    rows, cols, vals = [], [], []
    diag = np.zeros(ntot)
    bdir = np.zeros(ntot)
    for d in range(3):
        t1, t2 = (d + 1) % 3, (d + 2) % 3
        area = np.ones(n)
        shp1 = [1, 1, 1]
        shp1[t1] = n[t1]
        shp2 = [1, 1, 1]
        shp2[t2] = n[t2]
        area = area * h[t1].reshape(shp1) * h[t2].reshape(shp2)
        lamd = None if lam is None else np.asarray(lam[d], dtype=np.float64)
        periodic = bc[2 * d] == "periodic"
        for q in range(n[d] + 1):  # face below cell q (q = n: the top face)
            sl_face = [slice(None)] * 3
            sl_face[d] = slice(q, q + 1)
            lf = 1.0 if lamd is None else lamd[tuple(sl_face)]
            if 0 < q < n[d]:
                dc = abs(cc[d][q] - cc[d][q - 1])
                sl_p = [slice(None)] * 3
                sl_p[d] = slice(q - 1, q)
                sl_q = [slice(None)] * 3
                sl_q[d] = slice(q, q + 1)
                a = (area[tuple(sl_q)] / dc * lf).ravel()
                P, Q = idx[tuple(sl_p)].ravel(), idx[tuple(sl_q)].ravel()
                rows += [P, Q]
                cols += [Q, P]
                vals += [a, a]
                diag[P] -= a
                diag[Q] -= a
                continue
            side = 0 if q == 0 else 1
            cell = 0 if q == 0 else n[d] - 1
            sl_c = [slice(None)] * 3
            sl_c[d] = slice(cell, cell + 1)
            C = idx[tuple(sl_c)].ravel()
            if periodic:
                if q == n[d]:
                    continue  # the wrapped face is the q = 0 one
                dc = abs(0.5 * (h[d][0] + h[d][-1]))
                sl_o = [slice(None)] * 3
                sl_o[d] = slice(n[d] - 1, n[d])
                a = (area[tuple(sl_c)] / dc * lf).ravel()
                O = idx[tuple(sl_o)].ravel()
                rows += [C, O]
                cols += [O, C]
                vals += [a, a]
                diag[C] -= a
                diag[O] -= a
                continue
            kind = bc[2 * d + side]
            if kind == "Neumann":
                # gradient g: ghost = x + g * distance, b -= A_f g / delta
                bdir[C] -= (area[tuple(sl_c)] * lf).ravel() * values[2 * d + side]
                continue
            a = (area[tuple(sl_c)] / h[d][cell] * lf).ravel()
            diag[C] -= 2.0 * a
            bdir[C] -= 2.0 * a * values[2 * d + side]
    A = sp.csr_matrix((np.concatenate(vals) if vals else np.zeros(0),
                       (np.concatenate(rows) if rows else np.zeros(0, int),
                        np.concatenate(cols) if cols else np.zeros(0, int))), shape=(ntot, ntot))
    A = (A + sp.diags(diag)).tocsr()
    V = (h[0][:, None, None] * h[1][None, :, None] * h[2][None, None, :]).ravel()
    return A, V, bdir
