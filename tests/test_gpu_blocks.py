"""GPU parity of B, B^T, the Stokes block operator, the mass matrices and the
multigrid transfers against the oracle (FP64 within 1e-12 relative)."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import BC_COMBOS, consistent, rel_err, smooth_viscosity

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _pair(level):
    """oracle fine shell and its coarse (pressure) shell; device shell with both levels."""
    sh = O.Shell(level)
    return sh, sh.coarser(), T.Shell(level, num_levels=2)


@pytest.mark.parametrize("level", [2, 3, 4])
@pytest.mark.parametrize("bcs", BC_COMBOS)
def test_divergence_and_gradient(cuda, level, bcs):
    import torch

    sh, shc, g = _pair(level)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 3))
    p = consistent(shc, O.seeded_normal(shc.scalar_shape, 4))
    ob = O.Divergence(sh, bc_cmb=bcs[0], bc_surface=bcs[1])
    ref_b = ob.apply(u)
    ref_bt = ob.apply_transpose(p)
    B = T.Divergence(g, level=1, bc_cmb=bcs[0], bc_surface=bcs[1])
    BT = T.Gradient(g, level=1, bc_cmb=bcs[0], bc_surface=bcs[1])
    out_p = torch.full(shc.scalar_shape, float("nan"), dtype=torch.float64, device=cuda)
    B.apply(torch.tensor(u, device=cuda), out_p)
    out_u = torch.full(sh.vec_shape, float("nan"), dtype=torch.float64, device=cuda)
    BT.apply(torch.tensor(p, device=cuda), out_u)
    assert rel_err(out_p.cpu().numpy(), ref_b) < TOL64
    assert rel_err(out_u.cpu().numpy(), ref_bt) < TOL64


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2)])
def test_divergence_gradient_transpose(cuda, bcs):
    """p^T (B u) == u^T (B^T p) with owned-node dots (B and B^T are transposes)."""
    import torch

    level = 4
    sh, shc, g = _pair(level)
    u = torch.tensor(consistent(sh, O.seeded_normal(sh.vec_shape, 5)), device=cuda)
    p = torch.tensor(consistent(shc, O.seeded_normal(shc.scalar_shape, 6)), device=cuda)
    Bu = torch.zeros(shc.scalar_shape, dtype=torch.float64, device=cuda)
    BTp = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    T.Divergence(g, 1, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, Bu)
    T.Gradient(g, 1, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(p, BTp)
    a = g.dot(p, Bu, level=0)
    b = g.dot(u, BTp, level=1)
    assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2), (2, 2)])
def test_stokes_operator(cuda, bcs):
    import torch

    level = 3
    sh, shc, g = _pair(level)
    k = smooth_viscosity(sh, 7, 100.0)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 8))
    p = consistent(shc, O.seeded_normal(shc.scalar_shape, 9))
    A = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1])
    Bo = O.Divergence(sh, bc_cmb=bcs[0], bc_surface=bcs[1])
    ref_u = A.apply(u, path="slow") + Bo.apply_transpose(p)
    ref_p = Bo.apply(u)
    S = T.Stokes(g, level=1, k=torch.tensor(k, device=cuda), bc_cmb=bcs[0], bc_surface=bcs[1])
    src = [torch.tensor(u[c], device=cuda) for c in range(3)] + [torch.tensor(p, device=cuda)]
    dst = [torch.full_like(src[0], float("nan")) for _ in range(3)] + [torch.full_like(src[3], float("nan"))]
    S.apply(src, dst)
    got_u = np.stack([dst[c].cpu().numpy() for c in range(3)])
    assert rel_err(got_u, ref_u) < TOL64
    assert rel_err(dst[3].cpu().numpy(), ref_p) < TOL64


def test_mass_matrices(cuda):
    import torch

    level = 3
    sh = O.Shell(level)
    g = T.Shell(level)
    k = smooth_viscosity(sh, 10, 10.0)
    ref = O.kmass_lumped(sh, k)
    out = torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda)
    T.kmass_lumped_diagonal(g, 0, torch.tensor(k, device=cuda), out)
    assert rel_err(out.cpu().numpy(), ref) < TOL64
    v = consistent(sh, O.seeded_normal(sh.vec_shape, 11))
    ref = O.vector_mass(sh, v)
    outv = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    T.vector_mass_apply(g, 0, torch.tensor(v, device=cuda), outv)
    assert rel_err(outv.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("level", [2, 4, 5])
def test_transfers(cuda, level):
    import torch

    sh = O.Shell(level)
    shc = sh.coarser()
    g = T.Shell(level, num_levels=2)
    vc = consistent(shc, O.seeded_normal(shc.vec_shape, 12))
    vf = consistent(sh, O.seeded_normal(sh.vec_shape, 13))
    ref_p = O.prolongate_add(sh, vc.copy(), vf.copy())
    ref_r = O.restrict(sh, vf)
    fine = torch.tensor(vf, device=cuda)
    T.prolongate_add(g, 1, torch.tensor(vc, device=cuda), fine)
    coarse = torch.full(shc.vec_shape, float("nan"), dtype=torch.float64, device=cuda)
    T.restrict(g, 1, torch.tensor(vf, device=cuda), coarse)
    assert rel_err(fine.cpu().numpy(), ref_p) < 1e-14
    assert rel_err(coarse.cpu().numpy(), ref_r) < 1e-14


def test_f32_blocks(cuda):
    import torch

    level = 4
    sh, shc, g = _pair(level)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 14))
    ref = O.Divergence(sh, bc_cmb=1, bc_surface=2).apply(u)
    out = torch.zeros(shc.scalar_shape, dtype=torch.float32, device=cuda)
    T.Divergence(g, 1, dtype=torch.float32, bc_cmb=1, bc_surface=2).apply(torch.tensor(u, dtype=torch.float32, device=cuda), out)
    assert rel_err(out.double().cpu().numpy(), ref) < 1e-5
