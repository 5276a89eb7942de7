"""Seeded synthetic inputs for the Stokes workloads (no datasets are involved).

* viscosity: eta = exp(A * s(x_hat) * cos(pi (r - r_min) / (r_max - r_min))),
  s = sum of 8 real spherical harmonics of degree <= 4 with seeded (l, m, c),
  normalised to max |s| = 1 over the level's nodes; A = ln(10) gives a contrast
  of 10^2 (eta in [0.1, 10]). Real harmonics are the orthonormal ones built
  from the associated Legendre recursion (written here, not taken from the
  reference's SphericalHarmonicsTool).
* temperature: a smooth field of the same kind (8 harmonics times sin(pi
  (r - r_min) / (r_max - r_min))) plus N(0, 0.01) noise drawn per unique node.
* per-cell viscosity with blocks (adjoint workload): the smooth field above
  evaluated at cell centres times seeded piecewise-constant lateral blocks
  (tiles of each diamond, a seeded subset raised by a log-uniform factor in
  [1, 10^4]), all radii.
* buoyancy right-hand side f = M (T r_hat) with the vector mass matrix, then
  Dirichlet rows zeroed and free-slip normal components removed (the app's
  RHS assembly, apps/mantlecirculation/src/stokes_solver.hpp:650-671).

Every field is a function of the node's physical position (or of its
canonical node id for the noise), so interface duplicates are equal.
"""
from __future__ import annotations

import math

import numpy as np

import terra_b200 as T


def _assoc_legendre(lmax, x):
    """P_l^m(x) for 0 <= m <= l <= lmax (Condon-Shortley phase omitted)."""
    P = {}
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    P[(0, 0)] = np.ones_like(x)
    for m in range(1, lmax + 1):
        P[(m, m)] = (2 * m - 1) * s * P[(m - 1, m - 1)]
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * x * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * x * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    return P


def real_sh(l, m, xyz):
    """Orthonormal real spherical harmonic Y_lm at unit vectors xyz (..., 3)."""
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    phi = np.arctan2(y, x)
    P = _assoc_legendre(l, np.clip(z, -1.0, 1.0))
    am = abs(m)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    if m == 0:
        return norm * P[(l, 0)]
    if m > 0:
        return math.sqrt(2.0) * norm * P[(l, am)] * np.cos(am * phi)
    return math.sqrt(2.0) * norm * P[(l, am)] * np.sin(am * phi)


def _harmonic_sum(xhat, seed, terms=8, lmax=4):
    rng = np.random.default_rng(seed)
    s = np.zeros(xhat.shape[:-1])
    for _ in range(terms):
        l = int(rng.integers(1, lmax + 1))
        m = int(rng.integers(-l, l + 1))
        c = rng.standard_normal()
        s += c * real_sh(l, m, xhat)
    return s / np.abs(s).max()


def _geometry(shell: "T.Shell", level: int):
    coords = shell.coords(level)  # (10, nl, nl, 3) unit vectors
    radii = shell.radii(level)
    return coords, radii


def viscosity(shell: "T.Shell", level: int, seed: int = 1, log_amplitude: float = math.log(10.0)):
    """Nodal viscosity (10, nl, nl, nr) as a numpy array."""
    coords, radii = _geometry(shell, level)
    s = _harmonic_sum(coords, seed)  # (10, nl, nl)
    rad = np.cos(math.pi * (radii - radii[0]) / (radii[-1] - radii[0]))
    return np.exp(log_amplitude * s[..., None] * rad[None, None, None, :])


def temperature(shell: "T.Shell", level: int, seed: int = 2, noise: float = 0.01):
    """Temperature (10, nl, nl, nr): smooth harmonics plus N(0, noise^2) per unique node (device tensor)."""
    import torch

    coords, radii = _geometry(shell, level)
    s = _harmonic_sum(coords, seed)
    rad = np.sin(math.pi * (radii - radii[0]) / (radii[-1] - radii[0]))
    t = torch.tensor(s[..., None] * rad[None, None, None, :], device="cuda")
    # Box-Muller on two seeded uniform fields that agree on interface duplicates
    u = T.random_vector(shell, level, 2, seed * 1000003 + 17)
    u1 = (0.5 * (u[0] + 1.0)).clamp_min(1e-300)
    u2 = 0.5 * (u[1] + 1.0)
    t += noise * torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * u2)
    return t


def buoyancy_rhs(shell: "T.Shell", level: int, temp, bc_cmb: int, bc_surface: int):
    """f = M (T r_hat) with boundary rows enforced; (3, 10, nl, nl, nr) device tensor."""
    import torch

    coords, radii = _geometry(shell, level)
    n = torch.tensor(coords, device="cuda").permute(3, 0, 1, 2)  # (3, 10, nl, nl)
    src = (temp[None] * n[..., None]).contiguous()
    f = torch.zeros_like(src)
    T.vector_mass_apply(shell, level, src, f)
    return enforce_boundary(shell, level, f, bc_cmb, bc_surface)


def enforce_boundary(shell: "T.Shell", level: int, f, bc_cmb: int, bc_surface: int):
    """Zero the Dirichlet boundary rows and remove the free-slip normal components of every boundary carrying
    that condition (the library's assign-masked and free-slip projection kernels, tn_vec_assign_masked /
    tn_vec_freeslip_project: strong_algebraic_dirichlet_enforcement.hpp:114-123,
    strong_algebraic_freeslip_enforcement.hpp:22-38)."""
    for flag, bc in ((T.FLAG_CMB, bc_cmb), (T.FLAG_SURFACE, bc_surface)):
        if bc == T.DIRICHLET:
            T.vec_assign_masked(shell, level, f, flag, 0.0)
        elif bc == T.FREESLIP:
            T.vec_freeslip_project(shell, level, f, flag)
    return f


def cell_viscosity_blocks(shell: "T.Shell", level: int, seed: int = 3, tiles: int = 4, fraction: float = 0.3,
                          max_log10: float = 4.0, background_log_amplitude: float = math.log(10.0)):
    """Per-cell viscosity (10, nl-1, nl-1, nr-1): smooth background times lateral blocks."""
    coords, radii = _geometry(shell, level)
    nl, nr = coords.shape[1], radii.shape[0]
    # cell centres: mean of the 4 corner unit vectors (normalised) and of the two radii
    c = 0.25 * (coords[:, :-1, :-1] + coords[:, 1:, :-1] + coords[:, :-1, 1:] + coords[:, 1:, 1:])
    c /= np.linalg.norm(c, axis=-1, keepdims=True)
    rmid = 0.5 * (radii[:-1] + radii[1:])
    s = _harmonic_sum(c, seed)
    rad = np.cos(math.pi * (rmid - radii[0]) / (radii[-1] - radii[0]))
    eta = np.exp(background_log_amplitude * s[..., None] * rad[None, None, None, :])
    rng = np.random.default_rng(seed + 101)
    t = max(1, min(tiles, nl - 1))
    edge = (nl - 1) // t
    for d in range(10):
        for ix in range(t):
            for iy in range(t):
                if rng.uniform() < fraction:
                    f = 10.0 ** rng.uniform(0.0, max_log10)
                    eta[d, ix * edge:(ix + 1) * edge, iy * edge:(iy + 1) * edge, :] *= f
    return eta


def cell_viscosity_radial_jump(shell: "T.Shell", level: int, seed: int = 1, contrast: float = 1e3,
                               jump: float = 30.0, r_jump: float = 0.9):
    """Per-cell viscosity (10, nl-1, nl-1, nr-1) with max/min <= `contrast`: the
    spherical-harmonic field times a radial cosine (as `viscosity`) at the cell
    centres spanning a factor contrast/jump, multiplied by `jump` in the cells
    whose mid radius lies below `r_jump`."""
    coords, radii = _geometry(shell, level)
    c = 0.25 * (coords[:, :-1, :-1] + coords[:, 1:, :-1] + coords[:, :-1, 1:] + coords[:, 1:, 1:])
    c /= np.linalg.norm(c, axis=-1, keepdims=True)
    rmid = 0.5 * (radii[:-1] + radii[1:])
    s = _harmonic_sum(c, seed)
    rad = np.cos(math.pi * (rmid - radii[0]) / (radii[-1] - radii[0]))
    amp = 0.5 * math.log(contrast / jump)
    eta = np.exp(amp * s[..., None] * rad[None, None, None, :])
    eta *= np.where(rmid < r_jump, jump, 1.0)[None, None, None, :]
    return eta


def schur_coefficient_from_cells(shell: "T.Shell", velocity_level: int, eta_cell, mode: str = "inverse_mean"):
    """Nodal Schur-block coefficient k = 1/eta on the pressure level (velocity_level - 1) for a per-cell
    viscosity, from the fine cells touching each pressure node (over all copies of an interface node).

    mode "inverse_mean" (default): k = 1 / mean(eta). mode "mean_inverse": k = mean(1 / eta). The two differ
    where a node touches cells of very different viscosity: the first follows the stiff cells, the second the
    soft ones. With cell-wise jumps of 1e4 (log-uniform lateral blocks at level 5) the lumped-mass Schur block
    built from "inverse_mean" takes FGMRES(30) to 1e-4 in 192 iterations against 657 for "mean_inverse", and
    with FGMRES(128) to 1e-8 in 1247 iterations, where "mean_inverse" still stands at 2e-7 after 2000."""
    if mode not in ("inverse_mean", "mean_inverse"):
        raise ValueError(mode)
    nlf = eta_cell.shape[1] + 1
    nrf = eta_cell.shape[3] + 1
    val = eta_cell if mode == "inverse_mean" else 1.0 / eta_cell
    acc = np.zeros((10, nlf, nlf, nrf))
    cnt = np.zeros((10, nlf, nlf, nrf))
    for dx in (0, 1):
        for dy in (0, 1):
            for dr in (0, 1):
                acc[:, dx:nlf - 1 + dx, dy:nlf - 1 + dy, dr:nrf - 1 + dr] += val
                cnt[:, dx:nlf - 1 + dx, dy:nlf - 1 + dy, dr:nrf - 1 + dr] += 1.0
    cls, ncls = shell.duplicate_classes(velocity_level)
    flat_a = acc.reshape(10 * nlf * nlf, nrf)
    flat_c = cnt.reshape(10 * nlf * nlf, nrf)
    cl = cls.reshape(-1)
    for k in range(ncls):
        m = np.where(cl == k)[0]
        flat_a[m] = flat_a[m].sum(axis=0)
        flat_c[m] = flat_c[m].sum(axis=0)
    mean = flat_a.reshape(acc.shape) / flat_c.reshape(cnt.shape)
    node = 1.0 / mean if mode == "inverse_mean" else mean
    return np.ascontiguousarray(node[:, ::2, ::2, ::2])
