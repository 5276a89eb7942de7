"""GPU parity of the Galerkin coarse operators, the stored-matrix apply, the
multigrid hierarchy (inverse diagonals, power-iteration spectra, V-cycle) and
the Stokes FGMRES / velocity CG solves against the oracle.

Tolerances: matrices and applies 1e-12 relative (FP64); a V-cycle 1e-9 (the
coarsest CG stops on a 1e-6 tolerance, so rounding differences between the
two sides pass through up to 50 CG steps); FP32 V-cycle 1e-4; solves reach
the 1e-8 relative residual and agree with the oracle's FGMRES history.
"""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import BC_COMBOS, consistent, rel_err, smooth_viscosity

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


def _q0_field(sh, seed, contrast):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(0.0, np.log(contrast), size=sh.cell_shape))


@pytest.mark.parametrize("q0", [False, True])
def test_gca_matrices_match_oracle(cuda, q0):
    level = 3
    sh = O.Shell(level)
    shc = sh.coarser()
    g = T.Shell(level, num_levels=2)
    if q0:
        kc = _q0_field(sh, 3, 1e4)
        fo = O.EpsDivDiv(sh, k_q0=kc, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN)
        fine = T.EpsDivDiv(g, 1, k_cell=_t(kc), bc_cmb=T.NEUMANN, bc_surface=T.NEUMANN)
    else:
        k = smooth_viscosity(sh, 21, 100.0)
        fo = O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN)
        fine = T.EpsDivDiv(g, 1, k=_t(k), bc_cmb=T.NEUMANN, bc_surface=T.NEUMANN)
    ref = O.gca_coarsen(fo)
    coarse = T.EpsDivDiv(g, 0, k=_t(np.ones(shc.scalar_shape)))
    T.gca_build(fine, coarse)
    assert rel_err(coarse.local_matrices(), ref) < 1e-12


def test_gca_chain_from_stored_matrices(cuda):
    """level L-2 from the stored GCA matrices of level L-1 (gca.hpp with a
    stored fine operator)."""
    level = 3
    sh = O.Shell(level)
    s1 = sh.coarser()
    s0 = s1.coarser()
    g = T.Shell(level, num_levels=3)
    k = smooth_viscosity(sh, 22, 1000.0)
    m1 = O.gca_coarsen(O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN))
    m0 = O.gca_coarsen(O.EpsDivDiv(s1, k=np.ones(s1.scalar_shape), stored=m1), fine_mats=m1)
    fine = T.EpsDivDiv(g, 2, k=_t(k), bc_cmb=T.NEUMANN, bc_surface=T.NEUMANN)
    c1 = T.EpsDivDiv(g, 1, k=_t(np.ones(s1.scalar_shape)))
    c0 = T.EpsDivDiv(g, 0, k=_t(np.ones(s0.scalar_shape)))
    T.gca_build(fine, c1)
    T.gca_build(c1, c0)
    assert rel_err(c1.local_matrices(), m1) < 1e-12
    assert rel_err(c0.local_matrices(), m0) < 1e-12


@pytest.mark.parametrize("bcs", BC_COMBOS)
def test_stored_apply_matches_oracle(cuda, bcs):
    """Slow-path boundary treatment over stored matrices (Dirichlet masks,
    free-slip rotations; epsilon_divdiv_kerngen.hpp:1013-1242), apply and
    diagonal mode."""
    import torch

    level = 3
    sh = O.Shell(level)
    shc = sh.coarser()
    g = T.Shell(level, num_levels=2)
    k = smooth_viscosity(sh, 23, 100.0)
    mats = O.gca_coarsen(O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN))
    ref_op = O.EpsDivDiv(shc, k=np.ones(shc.scalar_shape), bc_cmb=bcs[0], bc_surface=bcs[1], stored=mats)
    fine = T.EpsDivDiv(g, 1, k=_t(k))
    coarse = T.EpsDivDiv(g, 0, k=_t(np.ones(shc.scalar_shape)), bc_cmb=bcs[0], bc_surface=bcs[1])
    T.gca_build(fine, coarse)
    u = consistent(shc, O.seeded_normal(shc.vec_shape, 24))
    out = torch.full(shc.vec_shape, float("nan"), dtype=torch.float64, device=cuda)
    coarse.apply(_t(u), out)
    assert rel_err(out.cpu().numpy(), ref_op.apply(u)) < 1e-12
    coarse.set_diagonal(True)
    coarse.apply(_t(u), out)
    assert rel_err(out.cpu().numpy(), ref_op.apply(u, diagonal=True)) < 1e-12
    # FP32 apply over the same matrices
    c32 = T.EpsDivDiv(g, 0, k=_t(np.ones(shc.scalar_shape), torch.float32), bc_cmb=bcs[0], bc_surface=bcs[1])
    T.gca_build(fine, c32)
    o32 = torch.zeros(shc.vec_shape, dtype=torch.float32, device=cuda)
    c32.apply(_t(u, torch.float32), o32)
    assert rel_err(o32.double().cpu().numpy(), ref_op.apply(u)) < 1e-5


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2), (2, 2)])
def test_stored_element_matrices_equal_matrix_free(cuda, bcs):
    """set_stored_matrix_mode(Full) on a level's own element matrices gives the
    matrix-free operator (the reference's slow == fast path)."""
    import torch

    level = 3
    sh = O.Shell(level)
    g = T.Shell(level)
    k = smooth_viscosity(sh, 25, 100.0)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 26))
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, path="slow")
    op = T.EpsDivDiv(g, 0, k=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1])
    op.set_stored_matrix_mode(T.STORED_FULL)
    out = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    op.apply(_t(u), out)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12
    op.set_stored_matrix_mode(T.STORED_OFF)
    op.apply(_t(u), out)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12


def test_random_vector_bit_exact(cuda):
    g = T.Shell(3, num_levels=2)
    for lvl, sh in ((1, O.Shell(3)), (0, O.Shell(2))):
        v = T.random_vector(g, lvl, 3, 4242).cpu().numpy()
        assert np.array_equal(v, O.seeded_uniform(sh, 3, 4242))


def _hierarchy(level, nlev, bcs, gca, seed=31, contrast=100.0, **opts):
    sh = O.Shell(level)
    k = smooth_viscosity(sh, seed, contrast)
    g = T.Shell(level, num_levels=nlev)
    solver = T.VelocitySolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=gca, **opts)
    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    o = solver.options
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=bool(gca), lambdas=lambdas,
                            cheb_order=o.chebyshev_order, cheb_iters=o.chebyshev_iterations,
                            coarse_max_iter=o.coarse_max_iterations, coarse_rtol=o.coarse_relative_tolerance,
                            coarse_atol=o.coarse_absolute_tolerance)
    return sh, k, g, solver, H


@pytest.mark.parametrize("gca", [1, 0])
def test_hierarchy_setup_matches_oracle(cuda, gca):
    """Coarse matrices, inverse diagonals and power-iteration spectra."""
    level, nlev = 3, 3
    sh, k, g, solver, H = _hierarchy(level, nlev, (1, 2), gca)
    for l in range(1, nlev):
        got = solver.inverse_diagonal(l).cpu().numpy()
        assert rel_err(got, H.inv_diag[l]) < 1e-12
        start = O.seeded_uniform(H.shells[l], 3, solver.options.seed + 7919 * l)
        lam = H.power_iteration(l, start, solver.options.power_iterations)
        assert abs(solver.level_lambda(l) - lam) <= 1e-10 * abs(lam)
    if gca:
        for l in range(nlev - 1):
            assert rel_err(solver.level_matrices(l), H.mats[l]) < 1e-12


@pytest.mark.parametrize("gca", [1, 0])
@pytest.mark.parametrize("bcs", [(1, 2), (1, 1)])
def test_vcycle_matches_oracle(cuda, gca, bcs):
    """One V-cycle with a converged coarsest solve: everything but the
    coarsest CG's stopping point is compared at 1e-9."""
    import torch

    level, nlev = 4, 3
    sh, k, g, solver, H = _hierarchy(level, nlev, bcs, gca, coarse_relative_tolerance=1e-13,
                                     coarse_max_iterations=3000)
    b = consistent(sh, O.seeded_normal(sh.vec_shape, 32))
    b = O.enforce_rhs_bcs(sh, b, bcs[0], bcs[1])
    ref = H.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    its, init, final = solver.coarse_stats()
    assert final <= 1e-13 * init


@pytest.mark.parametrize("bcs", [(1, 2), (1, 1)])
def test_vcycle_jacobi_smoother_matches_oracle(cuda, bcs):
    """One V-cycle with the damped Jacobi smoother (jacobi.hpp:51-60; 3 pre-
    and post-smoothing steps, omega = 0.8) and a converged coarsest solve,
    against the oracle at 1e-9."""
    import torch

    level, nlev = 4, 3
    sh, k, g, solver, H = _hierarchy(level, nlev, bcs, 1, smoother=T.SMOOTHER_JACOBI, jacobi_omega=0.8,
                                     chebyshev_iterations=3, coarse_relative_tolerance=1e-13,
                                     coarse_max_iterations=3000)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 35)), bcs[0], bcs[1])
    ref = H.multigrid(smoother="jacobi", omega=0.8).solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-9


@pytest.mark.parametrize("bcs", [(1, 2), (1, 1)])
def test_vcycle_reference_coarse_settings(cuda, bcs):
    """The reference's coarsest CG (50 iterations, 1e-6). On the level-2
    coarse problem 50 CG steps reduce the residual by only about 1e-3, and CG
    stopped that early amplifies rounding differences between the two sides
    (up to ~1e-4 observed); the converged-coarse test above carries the 1e-9
    parity, this one checks the reference settings end to end at 1e-3."""
    import torch

    level, nlev = 4, 3
    sh, k, g, solver, H = _hierarchy(level, nlev, bcs, 1)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 34)), bcs[0], bcs[1])
    ref = H.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-3
    its, init, final = solver.coarse_stats()
    assert 1 <= its <= 50 and (final <= 1e-6 * init or its == 50)


def test_vcycle_fp32(cuda):
    import torch

    level, nlev = 4, 3
    sh, k, g, solver, H = _hierarchy(level, nlev, (1, 2), 1, mixed_precision=1, coarse_relative_tolerance=1e-13,
                                     coarse_max_iterations=3000)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 33)), 1, 2)
    ref = H.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float32, device=cuda)
    solver.vcycle(x, _t(b, torch.float32))
    assert rel_err(x.double().cpu().numpy(), ref) < 1e-4


def _stokes_rhs(sh, seed, bcs):
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


def _stokes_vectors(sh, shp, f, cuda):
    import torch

    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [_t(f[c]) for c in range(3)] + [torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda)]
    return x, b


@pytest.mark.parametrize("gca", [1, 0])
def test_stokes_fgmres_matches_oracle(cuda, gca):
    """No-slip on both boundaries: the FGMRES residual history equals the
    oracle's step by step and the solutions agree."""
    level, nlev, bcs = 3, 3, (1, 1)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 41, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=gca, relative_tolerance=1e-8,
                            absolute_tolerance=0.0, normalize_pressure=0)
    f = _stokes_rhs(sh, 42, bcs)
    x, b = _stokes_vectors(sh, shp, f, cuda)
    assert solver.solve(x, b)
    its, rr, conv = solver.result()
    hist = solver.history()
    assert conv and rr <= 1e-8 and len(hist) == its + 1

    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=bool(gca), lambdas=lambdas)
    S = O.StokesSystem(sh, k, bcs[0], bcs[1], H)
    bflat = S.join(f, np.zeros(shp.scalar_shape))
    xg = S.join(np.stack([x[c].cpu().numpy() for c in range(3)]), x[3].cpu().numpy())
    r = bflat - S.apply(xg)
    assert np.sqrt(S.dot(r, r)) <= 1.0001e-8 * np.sqrt(S.dot(bflat, bflat))

    ohist = []
    xo, _ = O.fgmres(S.apply, np.zeros_like(bflat), bflat, S.dot, S.precondition, 30, 1e-8, 0.0, 300, ohist)
    assert len(ohist) == len(hist)
    assert np.allclose(hist, ohist, rtol=1e-5, atol=1e-13)
    uo, po = S.split(xo)
    ug, pg = S.split(xg)
    assert rel_err(ug, uo) < 1e-6
    own = shp.owned.astype(bool)
    assert rel_err(pg - pg[own].mean(), po - po[own].mean()) < 1e-5


def test_projected_stokes_fgmres_matches_oracle(cuda):
    """The benchmark's setting: free-slip surface with the pressure-mean projection (project_pressure_mean). The
    iteration runs on P K with the preconditioner P M, P removing the owned-node pressure mean from every
    entry; with a zero pressure right-hand side that is FGMRES on those operators from a projected initial guess.
    The history equals the oracle's step by step, and the projected and unprojected residuals agree."""
    level, nlev, bcs = 3, 3, (1, 2)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 44, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], relative_tolerance=1e-8,
                            absolute_tolerance=0.0, normalize_pressure=0, project_pressure_mean=1)
    f = _stokes_rhs(sh, 45, bcs)
    x, b = _stokes_vectors(sh, shp, f, cuda)
    assert solver.solve(x, b)
    its, rr, conv = solver.result()
    hist = solver.history()
    assert conv and rr <= 1e-8 and len(hist) == its + 1

    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=True, lambdas=lambdas)
    S = O.StokesSystem(sh, k, bcs[0], bcs[1], H)
    own = shp.owned.astype(bool)

    def proj(v):
        u, p = S.split(v)
        return S.join(u, p - p[own].sum() / own.sum())

    bflat = S.join(f, np.zeros(shp.scalar_shape))
    ohist = []
    xo, _ = O.fgmres(lambda v: proj(S.apply(v)), np.zeros_like(bflat), bflat, S.dot,
                     lambda v: proj(S.precondition(v)), 30, 1e-8, 0.0, 300, ohist)
    assert len(ohist) == len(hist)
    assert np.allclose(hist, ohist, rtol=1e-5, atol=1e-13)
    xg = S.join(np.stack([x[c].cpu().numpy() for c in range(3)]), x[3].cpu().numpy())
    uo, po = S.split(xo)
    ug, pg = S.split(xg)
    assert rel_err(ug, uo) < 1e-6
    assert rel_err(pg - pg[own].mean(), po - po[own].mean()) < 1e-5
    # the unprojected residual of the reference's system (full_residual) sits at the O(h^2) floor of the uniform
    # divergence part: above the projected tolerance, far below the right-hand side
    assert rr <= solver.full_residual() < 1e-4


def test_stokes_freeslip_solve(cuda):
    """Free-slip surface, no-slip CMB (the benchmark boundary conditions):
    reaches the 1e-8 relative residual measured with the oracle's operator,
    and the pressure leaves with zero owned-node mean."""
    level, nlev, bcs = 3, 3, (1, 2)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 48, 100.0)
    g = T.Shell(level, num_levels=nlev)
    f = _stokes_rhs(sh, 49, bcs)
    solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], absolute_tolerance=0.0,
                            normalize_pressure=0)
    x, b = _stokes_vectors(sh, shp, f, cuda)
    assert solver.solve(x, b)
    its, rr, conv = solver.result()
    assert conv and rr <= 1e-8
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=True, lambdas=[None] * nlev)
    S = O.StokesSystem(sh, k, bcs[0], bcs[1], H)
    bflat = S.join(f, np.zeros(shp.scalar_shape))
    xg = S.join(np.stack([x[c].cpu().numpy() for c in range(3)]), x[3].cpu().numpy())
    r = bflat - S.apply(xg)
    assert np.sqrt(S.dot(r, r)) <= 1.0001e-8 * np.sqrt(S.dot(bflat, bflat))
    # the same solve with the pressure normalisation of StokesContext::solve
    solver_n = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], absolute_tolerance=0.0)
    xn, bn = _stokes_vectors(sh, shp, f, cuda)
    assert solver_n.solve(xn, bn)
    pn = xn[3].cpu().numpy()
    own = shp.owned.astype(bool)
    assert abs(pn[own].mean()) <= 1e-12 * np.abs(pn).max()
    pg = x[3].cpu().numpy()
    assert rel_err(pn, pg - pg[own].mean()) < 1e-9


def test_stokes_preconditioner_matches_oracle(cuda):
    import torch

    level, nlev, bcs = 3, 3, (1, 2)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 43, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1])
    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=True, lambdas=lambdas)
    S = O.StokesSystem(sh, k, bcs[0], bcs[1], H)
    vu = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 44)), bcs[0], bcs[1])
    vp = consistent(shp, O.seeded_normal(shp.scalar_shape, 45))
    zu, zp = S.split(S.precondition(S.join(vu, vp)))
    v = [_t(vu[c]) for c in range(3)] + [_t(vp)]
    z = [torch.zeros_like(t) for t in v]
    solver.precondition(v, z)
    assert rel_err(np.stack([z[c].cpu().numpy() for c in range(3)]), zu) < 1e-9
    assert rel_err(z[3].cpu().numpy(), zp) < 1e-12


def _max_duplicate_spread(g, level, v):
    """Largest difference between copies of one node (v: (ncomp, 10, nl, nl, nr))."""
    cls, n = g.duplicate_classes(level)
    flat = cls.reshape(-1)
    vv = v.reshape(v.shape[0], -1, v.shape[-1])
    spread = 0.0
    for k in range(n):
        idx = np.where(flat == k)[0]
        spread = max(spread, float(np.abs(vv[:, idx] - vv[:, idx[:1]]).max()))
    return spread


def test_stokes_mixed_precision_reaches_tolerance(cuda):
    """FP32 V-cycle inside FP64 FGMRES reaches the same 1e-8 relative residual;
    the solution is compared with the FP64 solve. Both solutions hold bitwise
    equal values on every copy of an interface node (a solution used as the
    data of another solve, e.g. an adjoint right-hand side, must be consistent)."""
    import torch

    level, nlev, bcs = 4, 3, (1, 1)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 46, 100.0)
    f = _stokes_rhs(sh, 47, bcs)
    g = T.Shell(level, num_levels=nlev)
    sols = []
    for mixed in (0, 1):
        solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], mixed_precision=mixed,
                                absolute_tolerance=0.0)
        x, b = _stokes_vectors(sh, shp, f, cuda)
        assert solver.solve(x, b)
        its, rr, conv = solver.result()
        assert conv and rr <= 1e-8
        sols.append((np.stack([x[c].cpu().numpy() for c in range(3)]), x[3].cpu().numpy(), its))
        assert _max_duplicate_spread(g, nlev - 1, sols[-1][0]) == 0.0
        assert _max_duplicate_spread(g, nlev - 2, sols[-1][1][None]) == 0.0
    (u64, p64, it64), (u32, p32, it32) = sols
    assert it32 <= 1.25 * it64 + 5
    # both stop at a 1e-8 residual, so they agree to the problem's conditioning
    # times that tolerance: relative L2 over owned nodes, plus a max-norm bound
    ownu = sh.owned.astype(bool)
    l2 = np.sqrt(np.sum((u32 - u64)[:, ownu] ** 2) / np.sum(u64[:, ownu] ** 2))
    assert l2 < 1e-6
    assert rel_err(u32, u64) < 1e-5
    own = shp.owned.astype(bool)
    assert rel_err(p32 - p32[own].mean(), p64 - p64[own].mean()) < 1e-5


def test_velocity_cg_matches_oracle(cuda):
    """CG with the GMG preconditioner (Chebyshev order 3), Dirichlet on both
    boundaries, N(0,1) body force: the same iterates as the oracle's CG."""
    import torch

    level, nlev, bcs = 3, 3, (1, 1)
    sh, k, g, solver, H = _hierarchy(level, nlev, bcs, 1, contrast=10.0, chebyshev_order=3,
                                     relative_tolerance=1e-8, absolute_tolerance=0.0)
    f = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 51)), bcs[0], bcs[1])
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    assert solver.solve(x, _t(f))
    its, rr, conv = solver.result()
    hist = solver.history()
    mg = H.multigrid()
    A = lambda v: H.apply(len(H.shells) - 1, v)
    ohist = []
    xo = O.pcg(A, np.zeros(sh.vec_shape), f, sh.dot, 100, 1e-8, 0.0,
               precond=lambda z, r: mg.solve(np.zeros_like(r), r), history=ohist)
    assert len(ohist) == len(hist)
    assert np.allclose(hist, ohist, rtol=1e-6, atol=1e-13)
    assert rel_err(x.cpu().numpy(), xo) < 1e-7


@pytest.mark.parametrize("mixed", [1, 0])
def test_repeated_solves_stay_within_stated_drift(cuda, mixed):
    """The Galerkin stored apply and B's scatter add into their outputs with floating-point atomics, so two runs of
    the same solve need not agree bit for bit. The drift allowed between runs: the same iteration count, residual
    histories within 1e-4 relative with the FP32 V-cycle and 1e-8 in FP64, and solutions within 1e-10 and 1e-13
    relative (measured at levels 4 and 5: 1.1e-5 / 1.4e-12 mixed, 2e-10 / 1e-15 FP64)."""
    import torch

    from golden_inputs import stokes_rhs

    level, nlev = 4, 3
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 3, 100.0)
    f = stokes_rhs(sh, 4, (1, 2))
    g = T.Shell(level, num_levels=nlev)
    runs = []
    for _ in range(3):
        s = T.StokesSolver(g, eta=_t(k), bc_cmb=1, bc_surface=2, mixed_precision=mixed, relative_tolerance=1e-8,
                           absolute_tolerance=0.0, max_iterations=2000, project_pressure_mean=1,
                           coarse_solver=T.COARSE_DENSE)
        x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
        x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
        b = [_t(f[c]) for c in range(3)] + [torch.zeros_like(x[3])]
        assert s.solve(x, b)
        runs.append((np.array(s.history()), np.concatenate([t.cpu().numpy().ravel() for t in x[:3]])))
    h0, x0 = runs[0]
    for h, x in runs[1:]:
        assert len(h) == len(h0)
        assert np.allclose(h, h0, rtol=1e-4 if mixed else 1e-8, atol=0.0)
        assert rel_err(x, x0) < (1e-10 if mixed else 1e-13)
