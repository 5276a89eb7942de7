"""Seeded inputs of the golden fixtures (tests/golden/), shared by the generator and the tests.

Everything is derived from fixed seeds through numpy's PCG64 generator and the oracle's mesh, so the same
arrays come out on every host; ``checksum`` lets a test confirm that before comparing outputs.
"""
from __future__ import annotations

import numpy as np

import oracle as O
from helpers import BC_COMBOS, consistent, smooth_viscosity

BC_ALL = list(BC_COMBOS)
BC_L3 = [(1, 1), (1, 2), (2, 2)]

# the reference application's Stokes solve at level 3 (stokes_solver.hpp:169-691, GCA on all elements)
FGMRES_CASES = {
    "noslip": dict(level=3, num_levels=3, bcs=(1, 1), seed=41, max_it=200, rtol=1e-8),
    "freeslip": dict(level=3, num_levels=3, bcs=(1, 2), seed=48, max_it=60, rtol=1e-8),
}
POWER_SEED = 12345  # the product's default power-iteration seed; level l uses POWER_SEED + 7919 * l

# adaptive GCA (gca = 2): viscosity contrast 1e4 so that GCAElementsCollector marks part of the coarsest cells
SELECTIVE = dict(level=4, num_levels=3, seed=3, contrast=1e4, scale=1.0, bcs=(1, 1), fgmres_seed=4, max_it=30)
# The Stokes solve of the adaptive fixture: at contrast 1e4 the coarsest PCG(50, 1e-6) stops at its iteration
# limit, where two implementations' rounding drifts apart; contrast 10 scaled by 30 marks 94 of the 640 coarsest
# cells and the coarsest CG converges in about 35 iterations.
SELECTIVE_FGMRES = dict(level=4, num_levels=3, seed=3, contrast=10.0, scale=30.0, bcs=(1, 1), fgmres_seed=4,
                        max_it=40)
# (level, level_range, viscosity seed, contrast) of the marking fixtures
MARK_CASES = [(4, 2, 3, 1e4), (4, 3, 5, 3e3), (3, 2, 6, 1e4), (5, 3, 9, 1e5)]


def checksum(a) -> float:
    a = np.asarray(a, np.float64).ravel()
    w = np.sin(0.001 * np.arange(a.size) + 0.5)
    return float(np.dot(a, w))


def level_inputs(lat: int):
    sh = O.Shell(lat)
    c = sh.coarser()
    return dict(
        shell=sh,
        k=smooth_viscosity(sh, 7, 100.0),
        u=consistent(sh, O.seeded_normal(sh.vec_shape, 11)),
        p=consistent(c, O.seeded_normal(c.scalar_shape, 5)),
        k_q0=np.exp(np.random.default_rng(3).uniform(0.0, np.log(100.0), sh.cell_shape)),
        u_coarse=consistent(c, O.seeded_normal(c.vec_shape, 9)),
    )


def stokes_rhs(sh, seed, bcs):
    """Buoyancy-type right-hand side: vector mass of T(x) r_hat, boundary rows enforced."""
    rng = np.random.default_rng(seed)
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    Tf = np.zeros(X.shape[:-1])
    for _ in range(5):
        kv = rng.normal(size=3) * 2.0
        Tf += np.cos(X @ kv + rng.uniform(0, 2 * np.pi))
    Tf += 0.01 * rng.standard_normal(Tf.shape)
    Tf = consistent(sh, Tf)
    f = O.vector_mass(sh, np.moveaxis(Tf[..., None] * rhat, -1, 0))
    return O.enforce_rhs_bcs(sh, f, bcs[0], bcs[1])


def stokes_case(level, num_levels, bcs, seed, max_it, rtol):
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, seed, 100.0)
    f = stokes_rhs(sh, seed + 1, bcs)
    shells = [sh]
    for _ in range(num_levels - 1):
        shells.insert(0, shells[0].coarser())
    starts = [O.seeded_uniform(shells[l], 3, POWER_SEED + 7919 * l) for l in range(num_levels)]
    return dict(level=level, num_levels=num_levels, bcs=bcs, shell=sh, k=k, f=f,
                b=np.concatenate([f.ravel(), np.zeros(shp.scalar_shape).ravel()]),
                k_schur=1.0 / O.inject(shp, k), starts=starts, max_it=max_it, rtol=rtol)


def selective_case(c=None):
    """Inputs of the adaptive-GCA fixtures (SELECTIVE unless given): fine shell and viscosity, the injected
    viscosity of every coarser level (the rediscretised operators' coefficient), one seeded velocity per level,
    the Stokes right-hand side and the power-iteration start vectors."""
    c = SELECTIVE if c is None else c
    lat, nlev = c["level"], c["num_levels"]
    sh = O.Shell(lat)
    shp = sh.coarser()
    k = c["scale"] * smooth_viscosity(sh, c["seed"], c["contrast"])
    shells = [sh]
    for _ in range(nlev - 1):
        shells.insert(0, shells[0].coarser())
    k_levels = [None] * nlev
    k_levels[-1] = k
    for l in range(nlev - 2, -1, -1):
        k_levels[l] = O.inject(shells[l], k_levels[l + 1])
    u = [consistent(shells[l], O.seeded_normal(shells[l].vec_shape, 70 + l)) for l in range(nlev)]
    f = stokes_rhs(sh, c["fgmres_seed"], c["bcs"])
    starts = [O.seeded_uniform(shells[l], 3, POWER_SEED + 7919 * l) for l in range(nlev)]
    return dict(shell=sh, shells=shells, k=k, k_levels=k_levels, u=u, f=f, starts=starts,
                b=np.concatenate([f.ravel(), np.zeros(shp.scalar_shape).ravel()]),
                k_schur=1.0 / O.inject(shp, k), **c)
