"""Adjoint: the backward kernel against the oracle's FP64 restatement, and the
Stokes misfit gradient against central finite differences and the oracle's
FP64 adjoint (oracle FGMRES adjoint solve + oracle VJP).

Bars: VJP 1e-12 relative (FP64), 1e-5 (FP32); adjoint gradient vs central
differences 1e-6 relative (step 1e-5, forward solves to 1e-14: at step 1e-6
the FP64 rounding of J through the solves alone reaches ~1e-6 of the
difference quotient, at 1e-5 both it and the O(h^2) truncation stay below
1e-7); the GPU
adjoint state solves the oracle's adjoint system to 1e-12 and the oracle's
VJP at it reproduces the gradient to 1e-10."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import BC_COMBOS, consistent, rel_err

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


@pytest.mark.parametrize("bcs", BC_COMBOS)
def test_vjp_matches_oracle(cuda, bcs):
    import torch

    level = 3
    sh = O.Shell(level)
    rng = np.random.default_rng(70)
    kc = np.exp(rng.uniform(0.0, np.log(1e4), size=sh.cell_shape))
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 71))
    lam = consistent(sh, O.seeded_normal(sh.vec_shape, 72))
    ref_op = O.EpsDivDiv(sh, k_q0=kc, bc_cmb=bcs[0], bc_surface=bcs[1])
    ref = ref_op.vjp_logeta(u, lam)
    g = T.Shell(level)
    op = T.EpsDivDiv(g, 0, k_cell=_t(kc), bc_cmb=bcs[0], bc_surface=bcs[1])
    grad = torch.full(sh.cell_shape, float("nan"), dtype=torch.float64, device=cuda)
    gu = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    op.vjp(_t(u), _t(lam), grad, gu)
    assert rel_err(grad.cpu().numpy(), ref) < 1e-12
    assert rel_err(gu.cpu().numpy(), ref_op.apply(lam)) < 1e-12
    op32 = T.EpsDivDiv(g, 0, k_cell=_t(kc, torch.float32), bc_cmb=bcs[0], bc_surface=bcs[1])
    g32 = torch.zeros(sh.cell_shape, dtype=torch.float32, device=cuda)
    op32.vjp(_t(u, torch.float32), _t(lam, torch.float32), g32)
    assert rel_err(g32.double().cpu().numpy(), ref) < 1e-5


def _block_viscosity(sh, seed):
    rng = np.random.default_rng(seed)
    X = sh.physical_coords()
    c = 0.125 * sum(X[:, i:i + sh.nl - 1, j:j + sh.nl - 1, k:k + sh.nr - 1]
                    for i in (0, 1) for j in (0, 1) for k in (0, 1))
    eta = np.exp(0.5 * np.log(10.0) * np.sin(c @ np.array([1.1, -2.0, 0.7])))
    n = sh.nl - 1
    for d in range(10):
        for ix in range(2):
            for iy in range(2):
                if rng.uniform() < 0.5:
                    eta[d, ix * n // 2:(ix + 1) * n // 2, iy * n // 2:(iy + 1) * n // 2] *= 10 ** rng.uniform(0, 4)
    return eta


def _schur_k(sh, eta_cell):
    """1/eta at pressure nodes: mean of 1/eta over the fine cells touching the node, consistent on duplicates."""
    nlf, nrf = sh.nl, sh.nr
    acc = np.zeros(sh.scalar_shape)
    cnt = np.zeros(sh.scalar_shape)
    for dx in (0, 1):
        for dy in (0, 1):
            for dr in (0, 1):
                acc[:, dx:nlf - 1 + dx, dy:nlf - 1 + dy, dr:nrf - 1 + dr] += 1.0 / eta_cell
                cnt[:, dx:nlf - 1 + dx, dy:nlf - 1 + dy, dr:nrf - 1 + dr] += 1.0
    acc = sh.interface_sum(acc)
    cnt = sh.interface_sum(cnt)
    return np.ascontiguousarray((acc / cnt)[:, ::2, ::2, ::2])


def _forward(g, sh, shp, theta, ks, f, bcs, rtol, cuda):
    import torch

    solver = T.StokesSolver(g, eta_cell=_t(np.exp(theta)), k_schur=_t(ks), bc_cmb=bcs[0], bc_surface=bcs[1],
                            relative_tolerance=rtol, absolute_tolerance=0.0, max_iterations=8000,
                            project_pressure_mean=1, normalize_pressure=0)
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [_t(f[c]) for c in range(3)] + [torch.zeros_like(x[3])]
    assert solver.solve(x, b)
    return solver, x


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2)])
def test_stokes_misfit_gradient(cuda, bcs):
    """J = 1/2 sum_owned |u - u_obs|^2; dJ/dlog(eta_cell) by one adjoint solve
    + the backward kernel, against central differences along random
    directions and against the oracle's FP64 adjoint."""
    import torch

    level, nlev = 3, 3
    sh = O.Shell(level)
    shp = sh.coarser()
    g = T.Shell(level, num_levels=nlev)
    theta = np.log(_block_viscosity(sh, 80))
    ks = _schur_k(sh, np.exp(theta))
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    f = O.vector_mass(sh, np.moveaxis(np.cos(X @ np.array([1.5, -0.5, 1.0]))[..., None] * rhat, -1, 0))
    f = O.enforce_rhs_bcs(sh, f, bcs[0], bcs[1])
    rng = np.random.default_rng(81)
    theta_obs = theta + 0.1 * rng.standard_normal(theta.shape)
    _, x_obs = _forward(g, sh, shp, theta_obs, ks, f, bcs, 1e-14, cuda)
    u_obs = [x_obs[c] for c in range(3)]
    own = sh.owned.astype(bool)

    def J(th):
        _, x = _forward(g, sh, shp, th, ks, f, bcs, 1e-14, cuda)
        du = np.stack([(x[c] - u_obs[c]).cpu().numpy() for c in range(3)])
        return 0.5 * float(np.sum(du[:, own] ** 2))

    solver, x = _forward(g, sh, shp, theta, ks, f, bcs, 1e-14, cuda)
    grad = torch.zeros(sh.cell_shape, dtype=torch.float64, device=cuda)
    lam = [torch.zeros_like(t) for t in x]
    assert solver.misfit_gradient(x, u_obs, grad, lam)
    gnp = grad.cpu().numpy()
    h = 1e-5
    for _ in range(4):
        d = rng.standard_normal(theta.shape)
        fd = (J(theta + h * d) - J(theta - h * d)) / (2 * h)
        ad = float(np.sum(gnp * d))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)

    # oracle FP64 adjoint: the GPU adjoint state solves the oracle's (projected)
    # adjoint system, and the oracle VJP at it gives the gradient
    A = O.EpsDivDiv(sh, k_q0=np.exp(theta), bc_cmb=bcs[0], bc_surface=bcs[1])
    Bo = O.Divergence(sh, bc_cmb=bcs[0], bc_surface=bcs[1])
    ownp = shp.owned.astype(bool)
    xu = np.stack([x[c].cpu().numpy() for c in range(3)])
    lu = np.stack([lam[c].cpu().numpy() for c in range(3)])
    lp = lam[3].cpu().numpy()
    assert abs(lp[ownp].mean()) <= 1e-12 * np.abs(lp).max()
    rhs_u = O.enforce_rhs_bcs(sh, xu - np.stack([u_obs[c].cpu().numpy() for c in range(3)]), bcs[0], bcs[1])
    ru = rhs_u - A.apply(lu) - Bo.apply_transpose(lp)
    rp = -Bo.apply(lu)
    rp = rp - rp[ownp].mean()
    rel = np.sqrt(sh.dot(ru, ru) + shp.dot(rp, rp)) / np.sqrt(sh.dot(rhs_u, rhs_u))
    assert rel <= 1e-12
    g_ref = -A.vjp_logeta(xu, lu)
    assert rel_err(gnp, g_ref) < 1e-10
