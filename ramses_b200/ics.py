"""Seeded synthetic initial conditions for the hydro workloads.

Primitive fields are converted to conservative variables exactly as
``hydro/condinit.f90:36-57`` does (``u5 = 0 + ½ρu² + ½ρv² + ½ρw² + P/(γ-1)``,
evaluated in that order). Region-type ICs restate ``region_condinit``
(``hydro/init_flow_fine.f90:475-596``) for 'square' regions.

No public dataset is involved: every workload is a seeded synthetic field with
the shapes and value distributions of the configurations it stands in for.
"""
from __future__ import annotations

import numpy as np

from .mesh import Octree


def prim_to_cons(q: np.ndarray, gamma: float) -> np.ndarray:
    """q = (rho, u, v, w, P) [5, n] -> conservative [5, n] (condinit.f90:36-57)."""
    u = np.empty_like(q)
    u[0] = q[0]
    u[1] = q[0] * q[1]
    u[2] = q[0] * q[2]
    u[3] = q[0] * q[3]
    e = np.zeros_like(q[0])
    e = e + 0.5 * q[0] * q[1] ** 2
    e = e + 0.5 * q[0] * q[2] ** 2
    e = e + 0.5 * q[0] * q[3] ** 2
    e = e + q[4] / (gamma - 1.0)
    u[4] = e
    return u


def fill_all_levels(tree: Octree, prim_fn, gamma: float) -> np.ndarray:
    """uold[5, ncell] with every oct cell of every level set from
    ``prim_fn(x[n,3]) -> q[5,n]`` at cell centres (init_flow_fine style)."""
    u = np.zeros((5, tree.ncell))
    for l in range(1, tree.nlevelmax + 1):
        if tree.noct(l) == 0:
            continue
        cells, x = tree.cell_centres(l)
        u[:, cells - 1] = prim_to_cons(prim_fn(x), gamma)
    # coarse cell: mean of its oct (unused by the hydro path)
    return u


def sedov_prim(level: int, boxlen: float = 1.0, rho0: float = 1.0, p0: float = 1e-5,
               energy: float = 1.0, radius_cells: float = 2.5, gamma: float = 1.4,
               centre=(0.5, 0.5, 0.5)):
    """Sedov blast: ambient (rho0, v=0, p0); total energy ``energy`` spread
    uniformly as thermal energy over the cells of level ``level`` whose
    centre lies within ``radius_cells*dx`` of the centre (a 'square' region
    with exp_region=2, length=2*radius_cells*dx)."""
    dx = boxlen * 0.5 ** level
    n = 2 ** level
    c = np.asarray(centre) * boxlen
    # the cells within radius_cells of the centre lie in a window of
    # indices around it: count them there (same distance expression)
    lo = np.maximum(np.floor(c / dx - radius_cells - 2).astype(np.int64), 0)
    hi = np.minimum(np.ceil(c / dx + radius_cells + 2).astype(np.int64), n)
    ax = [(np.arange(lo[d], hi[d]) + 0.5) * dx for d in range(3)]
    X, Y, Z = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
    r = np.sqrt(((X - c[0]) / dx) ** 2 + ((Y - c[1]) / dx) ** 2 + ((Z - c[2]) / dx) ** 2)
    ncell = int(np.count_nonzero(r < radius_cells))
    p_in = (gamma - 1.0) * energy / (ncell * dx ** 3)

    def prim(x):
        rr = np.sqrt(((x[:, 0] - c[0]) / dx) ** 2 + ((x[:, 1] - c[1]) / dx) ** 2
                     + ((x[:, 2] - c[2]) / dx) ** 2)
        q = np.zeros((5, len(x)))
        q[0] = rho0
        q[4] = np.where(rr < radius_cells, p_in, p0)
        return q
    return prim


def shock_tube_prim(rho_l, p_l, u_l, rho_r, p_r, u_r, x0=0.5, boxlen=1.0, periodic_mirror=True):
    """Planar shock tube along x. With ``periodic_mirror`` the tube is
    [x0-L/2, x0+L/2) of a periodic box of length L: left state on
    x in [x0-L/2, x0), right on [x0, x0+L/2), so the second (wrapped)
    interface sits half a box away."""
    def prim(x):
        xs = x[:, 0] % boxlen
        left = xs < x0
        if periodic_mirror:
            left = ((xs - x0) % boxlen) >= boxlen / 2
        q = np.zeros((5, len(x)))
        q[0] = np.where(left, rho_l, rho_r)
        q[1] = np.where(left, u_l, u_r)
        q[4] = np.where(left, p_l, p_r)
        return q
    return prim


def _gaussian_field(n: int, rng, slope: float = -4.0):
    k = np.fft.fftfreq(n) * n
    kx, ky, kz = np.meshgrid(k, k, k[: n // 2 + 1], indexing="ij")
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    amp = np.zeros_like(kk)
    nz = kk > 0
    # P(k) ∝ k^slope for the 3D power spectrum; amplitude ∝ sqrt(P)
    amp[nz] = kk[nz] ** (slope / 2.0)
    return kx, ky, kz, amp


def turbulent_box_prim_grid(n: int, seed: int = 2024, mach: float = 5.0, sigma: float = 1.0,
                            p_over_rho: float = 0.01, gamma: float = 1.001, slope: float = -4.0):
    """Dense (n,n,n) [z,y,x] primitive arrays for the supersonic turbulent box:
    ln(rho) a Gaussian random field with P(k) ∝ k^-4 and std ``sigma``,
    rescaled to mean rho = 1; velocity a solenoidal Gaussian field with
    P(k) ∝ k^-4 rescaled to RMS Mach ``mach`` for c = sqrt(gamma*P/rho);
    P = p_over_rho * rho."""
    rng = np.random.default_rng(seed)
    kx, ky, kz, amp = _gaussian_field(n, rng, slope)
    shape = amp.shape

    def grf():
        re = rng.standard_normal(shape)
        im = rng.standard_normal(shape)
        f = np.fft.irfftn((re + 1j * im) * amp, s=(n, n, n), axes=(0, 1, 2))
        return f

    g = grf()
    g = (g - g.mean()) / g.std() * sigma
    rho = np.exp(g)
    rho /= rho.mean()
    # solenoidal velocity: project the Fourier modes onto k-perpendicular
    vh = []
    for _ in range(3):
        re = rng.standard_normal(shape)
        im = rng.standard_normal(shape)
        vh.append((re + 1j * im) * amp)
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    k2[k2 == 0] = 1.0
    kdotv = kx * vh[0] + ky * vh[1] + kz * vh[2]
    vh = [vh[0] - kx * kdotv / k2, vh[1] - ky * kdotv / k2, vh[2] - kz * kdotv / k2]
    v = [np.fft.irfftn(c, s=(n, n, n), axes=(0, 1, 2)) for c in vh]
    c_s = np.sqrt(gamma * p_over_rho)
    vrms = np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    scale = mach * c_s / vrms
    # irfftn axes are (x-index from kx, y, z): arrays are indexed [ix, iy, iz]
    q = np.stack([rho, v[0] * scale, v[1] * scale, v[2] * scale, p_over_rho * rho])
    return np.ascontiguousarray(q.transpose(0, 3, 2, 1))  # -> [var, z, y, x]


def fill_uniform_level_from_grid(tree: Octree, level: int, qgrid: np.ndarray, gamma: float,
                                 uold: np.ndarray | None = None) -> np.ndarray:
    """Set the cells of a complete level from dense [5, z, y, x] primitives and
    the coarser levels from their restriction (mean of the 8 children)."""
    if uold is None:
        uold = np.zeros((5, tree.ncell))
    idx = tree.cell_index(level)
    cons = prim_to_cons(qgrid.reshape(5, -1), gamma)
    uold[:, idx.reshape(-1) - 1] = cons
    cur = cons.reshape(5, *idx.shape)
    for l in range(level - 1, 0, -1):
        cur = 0.125 * (cur[:, 0::2, 0::2, 0::2] + cur[:, 1::2, 0::2, 0::2] + cur[:, 0::2, 1::2, 0::2]
                       + cur[:, 1::2, 1::2, 0::2] + cur[:, 0::2, 0::2, 1::2] + cur[:, 1::2, 0::2, 1::2]
                       + cur[:, 0::2, 1::2, 1::2] + cur[:, 1::2, 1::2, 1::2])
        uold[:, tree.cell_index(l).reshape(-1) - 1] = cur.reshape(5, -1)
    return uold


def blast_clumps_prim(n_clumps: int = 32, seed: int = 7, rho0: float = 1.0, p0: float = 1e-3,
                      contrast: float = 100.0, energy: float = 10.0, r_blast: float = 0.01,
                      gamma: float = 1.4):
    """Blast-clump stress test: ambient (rho0, p0); ``n_clumps`` seeded dense
    spheres (centres U[0.1,0.9]^3, radii U[0.01,0.05], density x contrast,
    pressure equilibrium); Sedov energy ``energy`` inside r_blast of the
    centre."""
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0.1, 0.9, size=(n_clumps, 3))
    rad = rng.uniform(0.01, 0.05, size=n_clumps)
    vol = 4.0 / 3.0 * np.pi * r_blast ** 3
    p_in = (gamma - 1.0) * energy / vol

    def prim(x):
        q = np.zeros((5, len(x)))
        q[0] = rho0
        q[4] = p0
        for c, r in zip(cen, rad):
            inside = np.sum((x - c) ** 2, axis=1) < r * r
            q[0][inside] = rho0 * contrast
        rb = np.sqrt(np.sum((x - 0.5) ** 2, axis=1))
        q[4] = np.where(rb < r_blast, p_in, q[4])
        return q
    return prim
