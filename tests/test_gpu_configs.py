"""The small workload configurations, through the C ABI.

Level-4 velocity problem: 17x17 nodes per diamond, 17 radial layers, Dirichlet
on both boundaries, seeded spherical-harmonic viscosity (amplitude ln 10) and
an N(0,1) body force; one operator apply against the oracle (1e-12) and a
CG solve preconditioned by the GMG V(2,2) with Chebyshev order 3 to 1e-8,
whose residual history equals the oracle's.

Adjoint with per-cell block viscosity: at level 4 with log-uniform [1, 10^2] lateral blocks in a smooth
background (contrast up to ~300), and at level 5 with [1, 10^4] blocks (configuration 3, contrast 8e4); J = 1/2
||u - u_obs||^2 with u_obs from a perturbed viscosity; the adjoint gradient against central differences along
random element directions to 1e-6 relative (level 4: step 1e-5, 3 directions; level 5: step 1e-6, 32 directions).
At the 10^4 contrast the solves use FGMRES(128) and the Schur coefficient 1/mean(eta) of the cells around each
pressure node, with which they reach 1e-13."""
import numpy as np
import pytest

import oracle as O
import synthetic as S
import terra_b200 as T
from helpers import consistent, rel_err

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


def test_level4_apply_and_velocity_cg(cuda):
    import torch

    level, nlev, bcs = 4, 3, (1, 1)
    sh = O.Shell(level)
    g = T.Shell(level, num_levels=nlev)
    fine = nlev - 1
    eta = S.viscosity(g, fine, seed=1)
    f = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 100)), *bcs)
    op = T.EpsDivDiv(g, fine, k=_t(eta), bc_cmb=bcs[0], bc_surface=bcs[1])
    out = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    op.apply(_t(f), out)
    assert rel_err(out.cpu().numpy(), O.EpsDivDiv(sh, k=eta, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(f)) < 1e-12

    solver = T.VelocitySolver(g, eta=_t(eta), bc_cmb=bcs[0], bc_surface=bcs[1], chebyshev_order=3,
                              chebyshev_iterations=2, relative_tolerance=1e-8, absolute_tolerance=0.0)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    assert solver.solve(x, _t(f))
    its, rr, conv = solver.result()
    hist = solver.history()
    assert conv and rr <= 1e-8
    o = solver.options
    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    H = O.VelocityHierarchy(sh, eta, bcs[0], bcs[1], nlev, gca=True, lambdas=lambdas, cheb_order=3, cheb_iters=2,
                            coarse_max_iter=o.coarse_max_iterations, coarse_rtol=o.coarse_relative_tolerance,
                            coarse_atol=o.coarse_absolute_tolerance)
    mg = H.multigrid()
    ohist = []
    xo = O.pcg(lambda v: H.apply(nlev - 1, v), np.zeros(sh.vec_shape), f, sh.dot, 200, 1e-8, 0.0,
               precond=lambda z, r: mg.solve(np.zeros_like(r), r), history=ohist)
    assert len(ohist) == len(hist)
    assert np.allclose(hist, ohist, rtol=1e-6, atol=1e-13)
    assert rel_err(x.cpu().numpy(), xo) < 1e-7


def test_block_viscosity_adjoint_gradient(cuda):
    import torch

    level, nlev, bcs = 4, 3, (1, 2)
    g = T.Shell(level, num_levels=nlev)
    fine = nlev - 1
    eta = S.cell_viscosity_blocks(g, fine, seed=3, tiles=4, fraction=0.3, max_log10=2.0,
                                  background_log_amplitude=0.25 * np.log(10.0))
    theta = np.log(eta)
    ks = S.schur_coefficient_from_cells(g, fine, eta)
    temp = S.temperature(g, fine, seed=4)
    f = S.buoyancy_rhs(g, fine, temp, *bcs)
    nlp, nrp = g.dims(fine - 1)
    rng = np.random.default_rng(5)
    theta_obs = theta + 0.1 * rng.standard_normal(theta.shape)
    k_schur = _t(ks)

    def forward(th):
        s = T.StokesSolver(g, eta_cell=_t(np.exp(th)), k_schur=k_schur, bc_cmb=bcs[0], bc_surface=bcs[1],
                           relative_tolerance=1e-13, absolute_tolerance=0.0, max_iterations=4000,
                           project_pressure_mean=1, normalize_pressure=0)
        x = [torch.zeros_like(f[0]) for _ in range(3)]
        x.append(torch.zeros((10, nlp, nlp, nrp), dtype=torch.float64, device=cuda))
        b = [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x[3])]
        assert s.solve(x, b)
        return s, x

    _, xo = forward(theta_obs)
    u_obs = [xo[c] for c in range(3)]
    own = torch.tensor(g.ownership(fine), device=cuda).bool()

    def J(th):
        _, x = forward(th)
        return 0.5 * float(sum(((x[c] - u_obs[c])[own] ** 2).sum() for c in range(3)))

    solver, x = forward(theta)
    grad = torch.zeros(theta.shape, dtype=torch.float64, device=cuda)
    assert solver.misfit_gradient(x, u_obs, grad)
    gnp = grad.cpu().numpy()
    h = 1e-5
    for _ in range(3):
        d = rng.standard_normal(theta.shape)
        fd = (J(theta + h * d) - J(theta - h * d)) / (2 * h)
        ad = float(np.sum(gnp * d))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_configuration3_adjoint_gradient_level5(cuda):
    """Configuration 3: level 5, per-cell viscosity from log-uniform [1, 1e4] lateral blocks in a smooth background
    (contrast 8e4), no-slip CMB / free-slip surface, J = 1/2 sum_owned |u - u_obs|^2. The forward and adjoint
    solves reach 1e-13 (FGMRES(128), Schur coefficient 1/mean(eta)), and the adjoint gradient agrees with central
    differences along 32 random element directions at step 1e-6 to 1e-6 relative. The perturbed solves start from
    the unperturbed solution and reduce their residual by 2e-9; the difference J(+) - J(-) is summed as
    1/2 (u+ - u-).(u+ + u- - 2 u_obs) with exact rounding (math.fsum), so no cancellation of two J values enters."""
    import math

    import torch

    level, nlev, bcs = 5, 4, (1, 2)
    g = T.Shell(level, num_levels=nlev)
    fine = nlev - 1
    eta = S.cell_viscosity_blocks(g, fine, seed=3, tiles=4, fraction=0.3, max_log10=4.0,
                                  background_log_amplitude=0.5 * np.log(10.0))
    assert eta.max() / eta.min() > 1e4
    theta = np.log(eta)
    ks = _t(S.schur_coefficient_from_cells(g, fine, eta))
    f = S.buoyancy_rhs(g, fine, S.temperature(g, fine, seed=2), *bcs)
    nlp, nrp = g.dims(fine - 1)
    own = torch.tensor(g.ownership(fine), device=cuda).bool()

    def solve(th, rtol, x0=None, max_iterations=4000):
        s = T.StokesSolver(g, eta_cell=_t(np.exp(th)), k_schur=ks, bc_cmb=bcs[0], bc_surface=bcs[1], restart=128,
                           coarse_solver=T.COARSE_DENSE, mixed_precision=1, relative_tolerance=rtol,
                           absolute_tolerance=0.0, max_iterations=max_iterations, project_pressure_mean=1,
                           normalize_pressure=0)
        x = [torch.zeros_like(f[0]) for _ in range(3)]
        x.append(torch.zeros((10, nlp, nlp, nrp), dtype=torch.float64, device=cuda))
        if x0 is not None:
            for t, t0 in zip(x, x0):
                t.copy_(t0)
        ok = s.solve(x, [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x[3])])
        return s, x, ok

    rng = np.random.default_rng(5)
    _, xo, ok = solve(theta + 0.1 * rng.standard_normal(theta.shape), 1e-10)
    assert ok
    u_obs = [xo[c] for c in range(3)]
    s, x_base, ok = solve(theta, 1e-13)
    assert ok
    grad = torch.zeros(theta.shape, dtype=torch.float64, device=cuda)
    assert s.misfit_gradient(x_base, u_obs, grad)
    assert s.result()[1] <= 1e-13
    gnp = grad.cpu().numpy()
    del s

    def delta_j(up, um):
        terms = [((up[c] - um[c]) * (up[c] + um[c] - 2 * u_obs[c]))[own].cpu().numpy() for c in range(3)]
        return 0.5 * math.fsum(np.concatenate(terms))

    h, errs = 1e-6, []
    drng = np.random.default_rng(6)
    for _ in range(32):
        d = drng.standard_normal(theta.shape)
        xs = []
        for sgn in (1.0, -1.0):
            _, x, ok = solve(theta + sgn * h * d, 2e-9, x_base, 3000)
            xs.append(x)
        fd = delta_j(xs[0], xs[1]) / (2 * h)
        ad = math.fsum((gnp * d).ravel())
        errs.append(abs(fd - ad) / abs(ad))
    assert max(errs) <= 1e-6, errs


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2), (2, 2)])
def test_129_radial_layers(cuda, bcs):
    """129 radial layers, as at level 7 (the radial kernel variant with four
    cells per lane), on a 9x9 lateral grid: operator applies in FP64 (1e-12) and
    FP32 (1e-5), B and B^T (1e-12), and a mixed-precision Stokes solve whose
    residual, recomputed with the oracle's operators, meets its tolerance. With
    free-slip on both boundaries the rigid rotations are a null space of the
    Stokes operator, which the solver does not remove, so that case checks the
    operators only."""
    import torch

    sh = O.Shell(3, 7)
    shp = sh.coarser()
    g = T.Shell(3, 7, num_levels=3)
    k = S.viscosity(g, 2, seed=6)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 60))
    p = consistent(shp, O.seeded_normal(shp.scalar_shape, 61))
    A = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1])
    ref = A.apply(u)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 1e-5)):
        op = T.EpsDivDiv(g, 2, k=_t(k, dt), bc_cmb=bcs[0], bc_surface=bcs[1])
        out = torch.full(sh.vec_shape, float("nan"), dtype=dt, device=cuda)
        op.apply(_t(u, dt), out)
        assert rel_err(out.double().cpu().numpy(), ref) < tol
    Bo = O.Divergence(sh, bc_cmb=bcs[0], bc_surface=bcs[1])
    out_p = torch.full(shp.scalar_shape, float("nan"), dtype=torch.float64, device=cuda)
    T.Divergence(g, 2, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(_t(u), out_p)
    assert rel_err(out_p.cpu().numpy(), Bo.apply(u)) < 1e-12
    out_u = torch.full(sh.vec_shape, float("nan"), dtype=torch.float64, device=cuda)
    T.Gradient(g, 2, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(_t(p), out_u)
    assert rel_err(out_u.cpu().numpy(), Bo.apply_transpose(p)) < 1e-12

    if bcs == (2, 2):
        return
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    f = O.vector_mass(sh, np.moveaxis(np.cos(X @ np.array([2.0, 1.0, -1.0]))[..., None] * rhat, -1, 0))
    f = O.enforce_rhs_bcs(sh, f, bcs[0], bcs[1])
    project = int(bcs[0] != 1 or bcs[1] != 1)
    solver = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], mixed_precision=1,
                            absolute_tolerance=0.0, max_iterations=3000, project_pressure_mean=project,
                            normalize_pressure=0)
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [_t(f[c]) for c in range(3)] + [torch.zeros_like(x[3])]
    assert solver.solve(x, b)
    xu = np.stack([x[c].cpu().numpy() for c in range(3)])
    xp = x[3].cpu().numpy()
    ru = f - A.apply(xu) - Bo.apply_transpose(xp)
    rp = -Bo.apply(xu)
    own = shp.owned.astype(bool)
    rp = rp - rp[own].mean()
    rel = np.sqrt(sh.dot(ru, ru) + shp.dot(rp, rp)) / np.sqrt(sh.dot(f, f))
    assert rel < 1.0001e-8, rel
