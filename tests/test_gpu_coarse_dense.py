"""The dense coarsest-level solve (coarse_solver = TN_COARSE_DENSE) and the multigrid used as a solver
(tn_multigrid_solver_create), against the oracle.

The dense option inverts the assembled coarsest operator once, so a V-cycle with it equals the oracle's V-cycle
with a converged coarsest CG (1e-9 relative, the bar of the converged-coarse V-cycle test). The multigrid solver
repeats V-cycles (Multigrid::solve_impl with statistics, multigrid.hpp:216-280): its residual history equals the
oracle's cycle by cycle at 1e-6.
"""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import consistent, rel_err, smooth_viscosity

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    t = torch.tensor(np.ascontiguousarray(a), device="cuda")
    return t if dtype is None else t.to(dtype)


def _oracle_hierarchy(sh, k, bcs, nlev, gca, solver, exact_coarse=True):
    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    o = solver.options
    kw = dict(coarse_rtol=1e-14, coarse_max_iter=5000) if exact_coarse else {}
    return O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=bool(gca), lambdas=lambdas,
                               cheb_order=o.chebyshev_order, cheb_iters=o.chebyshev_iterations, **kw)


@pytest.mark.parametrize("gca", [1, 0])
@pytest.mark.parametrize("bcs", [(1, 2), (1, 1)])
def test_vcycle_dense_coarse_equals_exact_coarse(cuda, gca, bcs):
    import torch

    level, nlev = 4, 3
    sh = O.Shell(level)
    k = smooth_viscosity(sh, 31, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.VelocitySolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=gca,
                              coarse_solver=T.COARSE_DENSE)
    H = _oracle_hierarchy(sh, k, bcs, nlev, gca, solver)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 32)), bcs[0], bcs[1])
    ref = H.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    # FP32 V-cycle around the FP64 dense coarse solve
    s32 = T.VelocitySolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=gca, mixed_precision=1,
                           coarse_solver=T.COARSE_DENSE)
    x32 = torch.zeros(sh.vec_shape, dtype=torch.float32, device=cuda)
    s32.vcycle(x32, _t(b, torch.float32))
    assert rel_err(x32.double().cpu().numpy(), ref) < 1e-4


@pytest.mark.parametrize("coarse", [T.COARSE_DENSE, T.COARSE_PCG])
def test_multigrid_solver_history_matches_oracle(cuda, coarse):
    import torch

    level, nlev, bcs = 4, 3, (1, 2)
    sh = O.Shell(level)
    k = smooth_viscosity(sh, 41, 100.0)
    g = T.Shell(level, num_levels=nlev)
    kw = dict(coarse_solver=coarse)
    if coarse == T.COARSE_PCG:
        kw.update(coarse_relative_tolerance=1e-14, coarse_max_iterations=5000)
    solver = T.MultigridSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], max_iterations=6,
                               relative_tolerance=1e-12, absolute_tolerance=0.0, **kw)
    H = _oracle_hierarchy(sh, k, bcs, nlev, 1, solver)
    mg = H.multigrid()
    A = H.ops[-1]
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 42)), *bcs)
    x = np.zeros(sh.vec_shape)
    r0 = np.sqrt(sh.dot(b, b))
    want = [1.0]
    for _ in range(6):
        x = mg.solve(x, b)
        r = b - A.apply(x)
        want.append(np.sqrt(sh.dot(r, r)) / r0)
    xs = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    bs = [_t(b[c]) for c in range(3)]
    solver.solve(xs, bs)
    hist = np.array(solver.history())
    assert len(hist) == 7
    assert np.allclose(hist, want, rtol=1e-6, atol=0.0)
    assert np.all(np.diff(hist) < 0) and hist[-1] < 0.1  # every V(2,2) cycle reduces the residual


@pytest.mark.parametrize("mixed", [0, 1])
def test_zero_start_vcycle_skips_first_apply_exactly(cuda, mixed):
    """The preconditioner starts its V-cycle from zero and writes the first pre-smoothing step's A x as zeros
    instead of applying A; tn_solver_vcycle on x = 0 applies A to the zeros. With GCA off and the dense coarsest
    solve no kernel on the path adds atomically, so the two results agree bit for bit (FP64, and the FP32 V-cycle
    of the mixed solver on the narrowed right-hand side)."""
    import torch

    level, nlev, bcs = 4, 3, (1, 2)
    sh = O.Shell(level)
    k = smooth_viscosity(sh, 51, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.VelocitySolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=0, mixed_precision=mixed,
                              coarse_solver=T.COARSE_DENSE)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 52)), *bcs)
    z = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.precondition(_t(b), z)
    dt = torch.float32 if mixed else torch.float64
    x = torch.zeros(sh.vec_shape, dtype=dt, device=cuda)
    solver.vcycle(x, _t(b, dt))
    assert float(z.abs().max()) > 0.0
    assert torch.equal(z, x.double())


def test_stokes_dense_coarse_reaches_tolerance(cuda):
    """The Stokes solve with the dense coarsest solve reaches 1e-8 and agrees with the reference-default
    (coarsest CG) solution."""
    import torch

    level, nlev, bcs = 4, 3, (1, 2)
    sh = O.Shell(level)
    shp = sh.coarser()
    k = smooth_viscosity(sh, 48, 100.0)
    g = T.Shell(level, num_levels=nlev)
    rng = np.random.default_rng(49)
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    f = O.vector_mass(sh, np.moveaxis(np.cos(X @ rng.normal(size=3))[..., None] * rhat, -1, 0))
    f = O.enforce_rhs_bcs(sh, f, *bcs)
    out = {}
    for name, coarse in (("dense", T.COARSE_DENSE), ("pcg", T.COARSE_PCG)):
        s = T.StokesSolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], coarse_solver=coarse,
                           project_pressure_mean=1, absolute_tolerance=0.0, max_iterations=500)
        x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
        x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
        b = [_t(f[c]) for c in range(3)] + [torch.zeros_like(x[3])]
        assert s.solve(x, b)
        its, rr, conv = s.result()
        assert conv and rr <= 1e-8
        out[name] = (np.stack([x[c].cpu().numpy() for c in range(3)]), its)
    assert rel_err(out["dense"][0], out["pcg"][0]) < 1e-6
    assert out["dense"][1] <= out["pcg"][1]


@pytest.mark.parametrize("gca", [1, 0])
def test_vcycle_linear_transfers_match_oracle(cuda, gca):
    """One V-cycle with the linear transfers (and, with GCA, linear interpolation in the Galerkin build),
    against the oracle's V-cycle with the same transfers and an exact coarsest solve."""
    import torch

    level, nlev, bcs = 4, 3, (1, 2)
    sh = O.Shell(level)
    k = smooth_viscosity(sh, 33, 100.0)
    g = T.Shell(level, num_levels=nlev)
    solver = T.VelocitySolver(g, eta=_t(k), bc_cmb=bcs[0], bc_surface=bcs[1], gca=gca,
                              coarse_solver=T.COARSE_DENSE, transfer=T.TRANSFER_LINEAR)
    lambdas = [None] + [solver.level_lambda(l) for l in range(1, nlev)]
    o = solver.options
    H = O.VelocityHierarchy(sh, k, bcs[0], bcs[1], nlev, gca=bool(gca), lambdas=lambdas,
                            cheb_order=o.chebyshev_order, cheb_iters=o.chebyshev_iterations, coarse_rtol=1e-14,
                            coarse_max_iter=5000, transfer="linear")
    if gca:
        for l in range(nlev - 1):
            assert rel_err(solver.level_matrices(l), H.mats[l]) < 1e-12
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 34)), *bcs)
    ref = H.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    solver.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-9


def test_gca_tensor_cores_equal_scalar(cuda):
    """The FP64 tensor-core triple products of the GCA build equal the scalar ones (1e-13) and the oracle's."""
    level = 4
    sh = O.Shell(level)
    k = smooth_viscosity(sh, 51, 1000.0)
    g = T.Shell(level, num_levels=2)
    fine = T.EpsDivDiv(g, 1, k=_t(k), bc_cmb=0, bc_surface=0)
    nc = sh.coarser().nl
    out = {}
    for tc in (True, False):
        coarse = T.EpsDivDiv(g, 0, k=_t(np.ones((10, nc, nc, nc))), bc_cmb=0, bc_surface=0)
        T.gca_build(fine, coarse, tensor_cores=tc)
        out[tc] = coarse.local_matrices()
    assert rel_err(out[True], out[False]) < 1e-13
    ref = O.gca_coarsen(O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN))
    assert rel_err(out[True], ref) < 1e-12
