"""GPU parity of the epsilon-div-div apply against the oracle.

Bar: FP64 within 1e-12 relative (max norm) of the oracle's reference slow path
(element matrices); FP32 within 2e-5 relative of the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import BC_COMBOS, consistent, rel_err, smooth_viscosity

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _setup(level, seed=0):
    sh = O.Shell(level)
    k = smooth_viscosity(sh, seed, contrast=100.0)
    u = consistent(sh, O.seeded_normal(sh.vec_shape, seed + 1))
    return sh, k, u


@pytest.mark.parametrize("level", [2, 3, 4])
@pytest.mark.parametrize("bcs", BC_COMBOS)
def test_apply_f64_matches_oracle(cuda, level, bcs):
    import torch

    sh, k, u = _setup(level, seed=level)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, path="slow")
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda), bc_cmb=bcs[0], bc_surface=bcs[1])
    src = torch.tensor(u, device=cuda)
    dst = torch.full_like(src, float("nan"))
    op.apply(src, dst)
    torch.cuda.synchronize()
    assert gsh.check_device_error() == 0
    assert rel_err(dst.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("level", [2, 4])
@pytest.mark.parametrize("bcs", BC_COMBOS)
def test_diagonal_f64_matches_oracle(cuda, level, bcs):
    import torch

    sh, k, u = _setup(level, seed=10 + level)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, path="slow", diagonal=True)
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda), bc_cmb=bcs[0], bc_surface=bcs[1], diagonal=True)
    dst = torch.zeros((3,) + sh.scalar_shape, dtype=torch.float64, device=cuda)
    op.apply(torch.tensor(u, device=cuda), dst)
    assert rel_err(dst.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("bcs", [(1, 1), (1, 2)])
def test_q0_coefficient(cuda, bcs):
    import torch

    level = 3
    sh = O.Shell(level)
    kq = np.exp(np.random.default_rng(5).uniform(0, np.log(1e4), sh.cell_shape))
    u = consistent(sh, O.seeded_normal(sh.vec_shape, 6))
    ref = O.EpsDivDiv(sh, k_q0=kq, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, path="slow")
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k_cell=torch.tensor(kq, device=cuda), bc_cmb=bcs[0], bc_surface=bcs[1])
    dst = torch.zeros((3,) + sh.scalar_shape, dtype=torch.float64, device=cuda)
    op.apply(torch.tensor(u, device=cuda), dst)
    assert rel_err(dst.cpu().numpy(), ref) < TOL64


def test_modes_add_and_skip_communication(cuda):
    """Replace+Skip leaves per-diamond partial sums; Add accumulates; the
    interface sum of the partial result equals the communicated apply."""
    import torch

    level = 3
    sh, k, u = _setup(level, seed=21)
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda))
    src = torch.tensor(u, device=cuda)
    full = torch.zeros_like(src)
    op.apply(src, full)
    op.set_modes(T.REPLACE, T.SKIP_COMMUNICATION)
    part = torch.zeros_like(src)
    op.apply(src, part)
    ref_part = O.EpsDivDiv(sh, k=k).apply(u, path="slow", comm=False)
    assert rel_err(part.cpu().numpy(), ref_part) < TOL64
    gsh.interface_sum(part)
    assert rel_err(part.cpu().numpy(), full.cpu().numpy()) < 1e-14
    op.set_modes(T.ADD, T.SKIP_COMMUNICATION)
    acc = torch.tensor(u, device=cuda)
    op.apply(src, acc)
    assert rel_err(acc.cpu().numpy(), u + ref_part) < TOL64


@pytest.mark.parametrize("tile", [(1, 1), (2, 3), (3, 5), (7, 9), (5, 64)])
def test_tile_shapes(cuda, tile):
    import torch

    level = 4
    sh, k, u = _setup(level, seed=31)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=1, bc_surface=2).apply(u, path="fast")
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda), bc_cmb=1, bc_surface=2)
    op.set_tile(*tile)
    dst = torch.zeros((3,) + sh.scalar_shape, dtype=torch.float64, device=cuda)
    op.apply(torch.tensor(u, device=cuda), dst)
    assert rel_err(dst.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("level", [5, 6])
def test_large_levels_f64(cuda, level):
    """Two and one radial cells per lane (levels 5/6) against the oracle fast path."""
    import torch

    sh, k, u = _setup(level, seed=41)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=1, bc_surface=2).apply(u, path="fast")
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda), bc_cmb=1, bc_surface=2)
    dst = torch.zeros((3,) + sh.scalar_shape, dtype=torch.float64, device=cuda)
    op.apply(torch.tensor(u, device=cuda), dst)
    assert rel_err(dst.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("level", [3, 5, 6])
@pytest.mark.parametrize("bcs", [(1, 1), (1, 2)])
def test_apply_f32(cuda, level, bcs):
    import torch

    sh, k, u = _setup(level, seed=51)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(u, path="fast")
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, dtype=torch.float32, device=cuda), bc_cmb=bcs[0], bc_surface=bcs[1])
    dst = torch.zeros((3,) + sh.scalar_shape, dtype=torch.float32, device=cuda)
    op.apply(torch.tensor(u, dtype=torch.float32, device=cuda), dst)
    assert rel_err(dst.cpu().numpy(), ref) < TOL32


def test_level7_consistency(cuda):
    """Four radial cells per lane (level 7): FP32 vs FP64 agreement and symmetry."""
    import torch

    level = 7
    gsh = T.Shell(level)
    nl, nr = gsh.dims()
    g = torch.Generator(device=cuda).manual_seed(3)
    k = torch.exp(0.3 * torch.randn((10, nl, nl, nr), generator=g, device=cuda, dtype=torch.float64))
    u = torch.randn((3, 10, nl, nl, nr), generator=g, device=cuda, dtype=torch.float64)
    v = torch.randn((3, 10, nl, nl, nr), generator=g, device=cuda, dtype=torch.float64)
    gsh.interface_sum(u)  # any assembled vectors will do
    gsh.interface_sum(v)
    op = T.EpsDivDiv(gsh, k=k)
    Au, Av = torch.zeros_like(u), torch.zeros_like(v)
    op.apply(u, Au)
    op.apply(v, Av)
    a, b = gsh.dot(v, Au), gsh.dot(u, Av)
    assert abs(a - b) <= 1e-10 * abs(a)
    op32 = T.EpsDivDiv(gsh, k=k.float())
    Au32 = torch.zeros_like(u, dtype=torch.float32)
    op32.apply(u.float(), Au32)
    assert rel_err(Au32.double().cpu().numpy(), Au.cpu().numpy()) < 1e-4


@pytest.mark.parametrize("level", [2, 4, 6])
def test_apply_is_deterministic(cuda, level):
    """No atomics: repeated applies are bitwise identical."""
    import torch

    sh, k, u = _setup(level, seed=61)
    gsh = T.Shell(level)
    op = T.EpsDivDiv(gsh, k=torch.tensor(k, device=cuda), bc_cmb=1, bc_surface=2)
    src = torch.tensor(u, device=cuda)
    first = torch.zeros_like(src)
    op.apply(src, first)
    for _ in range(20):
        again = torch.full_like(src, float("nan"))
        op.apply(src, again)
        assert torch.equal(again, first)
