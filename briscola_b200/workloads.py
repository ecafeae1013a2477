"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every right-hand side is generated from a seed.

* ``cavity(N)``  -- single brick N^3 on the unit cube, all walls (closed
  cavity), uniform spacing; RHS = discrete divergence of an N(0,1) face
  velocity field (wall-normal faces zero), volume-weighted zero mean.
* ``channel(N)`` -- N^3 on the unit cube, periodic x and z, walls in y with
  tanh clustering (gamma = 2); RHS = divergence of N(0,1) face velocities
  plus sin(2 pi x) cos(pi y) at the cell centres, zero mean.
* ``sphere(N)``  -- all walls, density 1 outside / 1000 inside a sphere of
  radius 0.2 at a seeded centre in [0.3,0.7]^3, VOF fraction from the signed
  distance ramped over 2 cells, face coefficient lambda = mean of 1/rho of the
  two cells; N(0,1) zero-mean RHS.

* ``multibrick(scale)`` -- seven axis-aligned bricks of uneven sizes
  (128x64x64, 96x96x96, 64x128x32, 128x32x64, 64x64x64, 48x96x48,
  32x32x128 cells) joined by cell-conforming contacts, Neumann outer walls,
  uniform spacing 1/128; every size and origin divided by ``scale`` (1, 2, 4
  or 8) for smaller cases.  N(0,1) cell RHS, volume-weighted zero mean.

Each returns (mesh, b, lam) with b the system right-hand side
b_sys = -V f of the reference (linearSystem.C:547-556) as a flat float64
array and lam None or the three face arrays.
"""
from __future__ import annotations

import numpy as np

from .mesh import NEUMANN, PERIODIC, Brick, Mesh, tanh_points, uniform_points


def face_divergence(brick: Brick, ux, uy, uz) -> np.ndarray:
    """Net outward flux of face velocities per cell (= V * div u)."""
    hx, hy, hz = (brick.cell_sizes(d) for d in range(3))
    ax = hy[:, None] * hz[None, :]
    ay = hx[:, None] * hz[None, :]
    az = hx[:, None] * hy[None, :]
    return ((ux[1:] - ux[:-1]) * ax[None] + (uy[:, 1:] - uy[:, :-1]) * ay[:, None, :]
            + (uz[:, :, 1:] - uz[:, :, :-1]) * az[:, :, None])


def random_face_velocity(brick: Brick, rng: np.random.Generator):
    n0, n1, n2 = brick.N
    per = brick.periodic
    u = []
    for d, shape in enumerate([(n0 + 1, n1, n2), (n0, n1 + 1, n2), (n0, n1, n2 + 1)]):
        a = rng.standard_normal(shape)
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[d] = 0
        sl_hi[d] = -1
        if per[d]:
            a[tuple(sl_hi)] = a[tuple(sl_lo)]  # the periodic face is one face
        else:
            a[tuple(sl_lo)] = 0.0
            a[tuple(sl_hi)] = 0.0
        u.append(a)
    return u


def zero_mean(f: np.ndarray, V: np.ndarray) -> np.ndarray:
    return f - (V * f).sum() / V.sum()


def cavity(N: int = 64, seed: int = 1000):
    br = Brick([uniform_points(N)] * 3, (NEUMANN,) * 6)
    rng = np.random.default_rng(seed)
    V = br.cell_volumes()
    flux = face_divergence(br, *random_face_velocity(br, rng))
    f = zero_mean(flux / V, V)
    return Mesh([br]), np.ascontiguousarray((-V * f).ravel()), None


def channel(N: int = 256, gamma: float = 2.0, seed: int = 2000):
    pts = [uniform_points(N), tanh_points(N, gamma), uniform_points(N)]
    br = Brick(pts, (PERIODIC, PERIODIC, NEUMANN, NEUMANN, PERIODIC, PERIODIC))
    rng = np.random.default_rng(seed)
    V = br.cell_volumes()
    flux = face_divergence(br, *random_face_velocity(br, rng))
    xc = br.cell_centres(0)[:, None, None]
    yc = br.cell_centres(1)[None, :, None]
    f = flux / V + np.sin(2 * np.pi * xc) * np.cos(np.pi * yc) * np.ones((1, 1, N))
    f = zero_mean(f, V)
    return Mesh([br]), np.ascontiguousarray((-V * f).ravel()), None


def sphere_lambda(brick: Brick, centre, radius=0.2, rho_in=1000.0, rho_out=1.0, ramp_cells=2.0):
    xc, yc, zc = (brick.cell_centres(d) for d in range(3))
    h = min(float(np.min(brick.cell_sizes(d))) for d in range(3))
    dist = np.sqrt((xc[:, None, None] - centre[0]) ** 2 + (yc[None, :, None] - centre[1]) ** 2
                   + (zc[None, None, :] - centre[2]) ** 2) - radius
    alpha = np.clip(0.5 - dist / (ramp_cells * h), 0.0, 1.0)
    rho = alpha * rho_in + (1.0 - alpha) * rho_out
    inv = 1.0 / rho
    n0, n1, n2 = brick.N
    lx = np.empty((n0 + 1, n1, n2))
    ly = np.empty((n0, n1 + 1, n2))
    lz = np.empty((n0, n1, n2 + 1))
    lx[1:-1] = 0.5 * (inv[1:] + inv[:-1])
    lx[0], lx[-1] = inv[0], inv[-1]
    ly[:, 1:-1] = 0.5 * (inv[:, 1:] + inv[:, :-1])
    ly[:, 0], ly[:, -1] = inv[:, 0], inv[:, -1]
    lz[:, :, 1:-1] = 0.5 * (inv[:, :, 1:] + inv[:, :, :-1])
    lz[:, :, 0], lz[:, :, -1] = inv[:, :, 0], inv[:, :, -1]
    return [np.ascontiguousarray(a) for a in (lx, ly, lz)]


def sphere(N: int = 256, seed: int = 4000):
    br = Brick([uniform_points(N)] * 3, (NEUMANN,) * 6)
    rng = np.random.default_rng(seed)
    centre = rng.uniform(0.3, 0.7, size=3)
    lam = sphere_lambda(br, centre)
    V = br.cell_volumes()
    f = zero_mean(rng.standard_normal(br.N), V)
    return Mesh([br]), np.ascontiguousarray((-V * f).ravel()), lam


# (cells, origin) of the seven bricks, in cells of spacing 1/128; origins are
# multiples of 16 so that the bricks coarsen together four times
MULTIBRICK_LAYOUT = [
    ((128, 64, 64), (0, 0, 0)),
    ((96, 96, 96), (128, 0, 0)),
    ((64, 128, 32), (0, 64, 0)),
    ((128, 32, 64), (0, 192, 0)),
    ((64, 64, 64), (224, 0, 0)),
    ((48, 96, 48), (64, 64, 0)),
    ((32, 32, 128), (0, 0, 64)),
]


def multibrick(scale: int = 1, seed: int = 3000):
    h = scale / 128.0
    bricks = []
    for n, o in MULTIBRICK_LAYOUT:
        n = tuple(v // scale for v in n)
        o = tuple(v // scale for v in o)
        pts = [o[d] * h + h * np.arange(n[d] + 1, dtype=np.float64) for d in range(3)]
        bricks.append(Brick(pts, (NEUMANN,) * 6, o))
    rng = np.random.default_rng(seed)
    f = [rng.standard_normal(br.N) for br in bricks]
    V = [br.cell_volumes() for br in bricks]
    mean = sum((v * a).sum() for v, a in zip(V, f)) / sum(v.sum() for v in V)
    b = np.concatenate([(-v * (a - mean)).ravel() for v, a in zip(V, f)])
    return Mesh(bricks), np.ascontiguousarray(b), None


CONFIGS = {"cavity": cavity, "channel": channel, "sphere": sphere, "multibrick": multibrick}


# ---------------------------------------------------------------------------
# time sequence of right-hand sides for the learned initial guess
# ---------------------------------------------------------------------------
class TaylorGreenSequence:
    """Right-hand sides b_t = -V div(u_t) on the all-wall unit cube (N^3,
    uniform): u_0 is the Taylor-Green field (sin pi x cos pi y cos pi z,
    -cos pi x sin pi y cos pi z, 0) on the cell faces (amplitude 1, zero
    normal velocity at the walls) plus seeded N(0, noise^2) on the interior
    faces; every step applies a fixed explicit update -- forward-Euler
    upwind advection by the constant velocity U0 plus diffusion nu -- and
    re-imposes zero wall-normal velocity.  Computed in FP64 on a torch
    device (synthetic data generation, not part of the solve)."""

    def __init__(self, N: int, seed: int, device, noise: float = 0.1, dt: float = 1e-3,
                 nu: float = 2e-4, U0=(1.0, 0.5, 0.25)):
        import torch

        self.torch = torch
        self.N = N
        self.h = 1.0 / N
        self.dt, self.nu, self.U0 = dt, nu, U0
        g = torch.Generator(device="cpu").manual_seed(seed)
        h = self.h
        c = (torch.arange(N, dtype=torch.float64) + 0.5) * h      # cell centres
        f = torch.arange(N + 1, dtype=torch.float64) * h           # face positions
        pi = np.pi
        ux = torch.sin(pi * f)[:, None, None] * torch.cos(pi * c)[None, :, None] * torch.cos(pi * c)[None, None, :]
        uy = -torch.cos(pi * c)[:, None, None] * torch.sin(pi * f)[None, :, None] * torch.cos(pi * c)[None, None, :]
        uz = torch.zeros(N, N, N + 1, dtype=torch.float64)
        u = [ux, uy, uz]
        for d in range(3):
            u[d] = u[d] + noise * torch.randn(u[d].shape, generator=g, dtype=torch.float64)
        self.u = [a.to(device) for a in u]
        self._walls()

    def _walls(self):
        for d in range(3):
            idx = [slice(None)] * 3
            idx[d] = 0
            self.u[d][tuple(idx)] = 0.0
            idx[d] = -1
            self.u[d][tuple(idx)] = 0.0

    def rhs(self):
        """b = -V div(u) of the current field, flat FP64 (k fastest)"""
        h = self.h
        ux, uy, uz = self.u
        div_flux = ((ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])) * h * h
        return (-div_flux).reshape(-1).contiguous()

    def step(self):
        torch = self.torch
        h, dt, nu = self.h, self.dt, self.nu
        new = []
        for a in self.u:
            lap = torch.zeros_like(a)
            adv = torch.zeros_like(a)
            for ax in range(3):
                lo = torch.cat([a.narrow(ax, 0, 1), a.narrow(ax, 0, a.shape[ax] - 1)], dim=ax)
                hi = torch.cat([a.narrow(ax, 1, a.shape[ax] - 1), a.narrow(ax, a.shape[ax] - 1, 1)], dim=ax)
                lap += (lo - 2 * a + hi) / (h * h)
                adv += self.U0[ax] * (a - lo) / h      # upwind, U0 > 0
            new.append(a + dt * (nu * lap - adv))
        self.u = new
        self._walls()
