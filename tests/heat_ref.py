"""Checkers of the direct heat solve, built on the oracle's Jacobi sweep (the restatement of
kernelHeatEquationTopOpen / OvenSurrounded, Tfield.h:93-240, pinned against the reference's
own thermal outputs).

`fixed_point` makes no use of the separable structure: it applies the oracle's sweep to unit
vectors to get the sweep as an affine map T -> M T + c over the voxels it updates, and solves
(I - M) T = c densely.  `separable_solve` restates the library's direct algorithm in numpy on
the library's one-dimensional modes, so that the CPU suite checks the Kronecker-sum form of the
reference's coefficients without a GPU."""
from __future__ import annotations

import numpy as np

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O


def initial_temperature(p: P.ShgParams) -> np.ndarray:
    """T = temp, the Dirichlet faces at t_peltier (Solver.h:319-323), shape (nz, n, n)."""
    n, nz = p.nx, p.nz
    T = np.full((nz, n, n), p.temp, dtype=np.float64)
    T[:, :, :] = p.temp
    fixed = dirichlet_mask(p)
    T[fixed] = p.t_peltier
    return T


def dirichlet_mask(p: P.ShgParams) -> np.ndarray:
    """Voxels no sweep writes: y = 0 (TOP_OPEN) or the four lateral faces (OVEN_SURROUNDED)."""
    n, nz = p.nx, p.nz
    m = np.zeros((nz, n, n), dtype=bool)
    if p.boundary == P.SHG_BOUNDARY_TOP_OPEN:
        m[:, 0, :] = True
    else:
        m[:, 0, :] = m[:, -1, :] = True
        m[:, :, 0] = m[:, :, -1] = True
    return m


def fixed_point(p: P.ShgParams, T0: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """The fixed point of the oracle's FP64 Jacobi sweep for heat source Q, with T0's Dirichlet
    voxels; dense, for grids of a few thousand voxels."""
    fixed = dirichlet_mask(p)
    free = np.flatnonzero(~fixed.ravel())
    base = np.where(fixed, T0, 0.0)
    c = O.jacobi_sweep(p, base.copy(), Q).ravel()[free]
    M = np.empty((free.size, free.size))
    for col, f in enumerate(free):
        t = base.copy().ravel()
        t[f] = 1.0
        M[:, col] = O.jacobi_sweep(p, t.reshape(base.shape), Q).ravel()[free] - c
    sol = np.linalg.solve(np.eye(free.size) - M, c)
    out = base.copy().ravel()
    out[free] = sol
    return out.reshape(T0.shape)


def separable_solve(p: P.ShgParams, T0: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """The library's direct algorithm in numpy: right-hand side of the scaled system, modes
    along x and y (shg_heat_operator_modes), a dense solve along z per mode, back."""
    n, nz = p.nx, p.nz
    dx, dy, dz = p.lx / (p.nx - 1), p.ly / (p.ny - 1), p.lz / (p.nz - 1)
    K, h, tinf = p.kappa, p.h_conv, p.t_inf
    bix, biy, biz = h * dx / K, h * dy / K, h * dz / K
    if p.boundary == P.SHG_BOUNDARY_TOP_OPEN:
        x0, mx, xr = 0, n, (1, 1)
        y0, my, yr = 1, n - 1, (0, 1)
    else:
        x0, mx, xr = 1, n - 2, (0, 0)
        y0, my, yr = 1, n - 2, (0, 0)
    X = np.arange(x0, x0 + mx)
    Y = np.arange(y0, y0 + my)
    Z = np.arange(nz)
    b = np.zeros((nz, my, mx))
    inner = ((Z[:, None, None] > 0) & (Z[:, None, None] < nz - 1) & (Y[None, :, None] > 0) &
             (Y[None, :, None] < n - 1) & (X[None, None, :] > 0) & (X[None, None, :] < n - 1))
    b += np.where(inner, Q[np.ix_(Z, Y, X)] / K, 0.0)
    for end, robin, idx in ((0, xr[0], x0 - 1), (mx - 1, xr[1], x0 + mx)):
        b[:, :, end] += 2 * bix * tinf / dx**2 if robin else T0[np.ix_(Z, Y, [idx])][:, :, 0] / dx**2
    for end, robin, idx in ((0, yr[0], y0 - 1), (my - 1, yr[1], y0 + my)):
        b[:, end, :] += 2 * biy * tinf / dy**2 if robin else T0[np.ix_(Z, [idx], X)][:, 0, :] / dy**2
    b[0] += 2 * biz * tinf / dz**2
    b[-1] += 2 * biz * tinf / dz**2
    lx, Fx, Gx = shg.heat_operator_modes(mx, dx, *xr, bix)
    ly, Fy, Gy = shg.heat_operator_modes(my, dy, *yr, biy)
    bh = np.einsum("ki,zji->zjk", Fx, b)
    bh = np.einsum("kj,zjx->zkx", Fy, bh)
    Az = np.diag(np.full(nz, 2.0)) - np.diag(np.ones(nz - 1), 1) - np.diag(np.ones(nz - 1), -1)
    Az[0, 0] = Az[-1, -1] = 2 * (1 + biz)
    Az[0, 1] = Az[-1, -2] = -2.0
    Az /= dz**2
    v = np.empty_like(bh)
    for j in range(my):
        for i in range(mx):
            v[:, j, i] = np.linalg.solve(Az + (lx[i] + ly[j]) * np.eye(nz), bh[:, j, i])
    v = np.einsum("jk,zkx->zjx", Gy, v)
    v = np.einsum("ik,zjk->zji", Gx, v)
    out = T0.copy()
    out[np.ix_(Z, Y, X)] = v
    return out


def small_case(n: int, nz: int, boundary: int, precision: int = 64, seed: int = 0):
    """A small thermal grid with a random positive heat source of a few kelvin's effect."""
    p = P.workload(n, nz, 4000.0, 20.0, 25.0, 2000.0, 30.0, precision=precision, thermal=1)
    p.boundary = boundary
    p.t_peltier = 40.0
    rng = np.random.default_rng(seed)
    L2 = p.lx * p.lx
    Q = rng.uniform(0.0, 1.0, (nz, n, n)) * 60.0 * p.kappa / L2
    return p, initial_temperature(p), Q
