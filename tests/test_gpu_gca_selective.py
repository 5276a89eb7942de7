"""Adaptive GCA (gca = 2) and the fast GCA build on the GPU, against the reference and the oracle.

tn_gca_mark_elements must reproduce the reference's GCAElementsCollector marks exactly. The selective coarse
operators (stored Galerkin matrices on the marked cells, the matrix-free operator of the injected viscosity
elsewhere) must apply as the reference's OperatorStoredMatrixMode::Selective operators do (1e-12), through the
solver hierarchy and through the operator-level API; the Stokes solve with gca = 2 follows the reference's
residual history (1e-5, as the other FGMRES fixtures). The fast build (rank form over on-the-fly matrices,
FP64 tensor-core triple products over stored ones) equals the plain scalar build to 1e-13. The FP32 V-cycle
over GCA levels with free slip on both boundaries (null-space penalty in FP32) stays within 1e-4 of the FP64
one.
"""
import os

import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from golden_inputs import BC_L3, MARK_CASES, SELECTIVE_FGMRES, checksum, selective_case
from helpers import consistent, rel_err, smooth_viscosity

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gca_selective.npz")


def _t(a, dtype=None):
    import torch

    t = torch.tensor(np.ascontiguousarray(a), device="cuda")
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def case():
    return selective_case()


@pytest.mark.parametrize("mc", MARK_CASES)
def test_marks_equal_reference(cuda, golden, mc):
    lat, lr, seed, contrast = mc
    sh = O.Shell(lat)
    g = T.Shell(lat, num_levels=lr + 1)
    marks = T.gca_mark_elements(g, lr, lr, _t(smooth_viscosity(sh, seed, contrast)))
    assert np.array_equal(marks.cpu().numpy(), golden[f"marks_L{lat}_r{lr}_s{seed}"])


@pytest.mark.parametrize("bc", BC_L3)
def test_solver_hierarchy_matches_reference(cuda, golden, case, bc):
    """Coarse levels of the gca = 2 hierarchy: the effective element matrices equal the oracle's, the stored
    cells are exactly the descendants of marked cells, and the smoother's inverse diagonal on level 1 is the
    reference's diagonal inverted."""
    import torch

    lat, nlev = case["level"], case["num_levels"]
    g = T.Shell(lat, num_levels=nlev)
    s = T.VelocitySolver(g, eta=_t(case["k"]), bc_cmb=bc[0], bc_surface=bc[1], gca=2, coarse_solver=T.COARSE_DENSE)
    H = O.VelocityHierarchy(case["shell"], case["k"], bc[0], bc[1], nlev, gca=2, lambdas=[None] + [1.0] * (nlev - 1))
    for l in range(nlev - 1):
        assert rel_err(s.level_matrices(l), H.mats[l]) < 1e-12
    marked1 = int(O.expand_marks(H.marks, 1).sum())
    cells1, bytes1 = s.level_storage(1)
    assert cells1 == marked1 and 0 < cells1 < int(np.prod(case["shells"][1].cell_shape))
    full = T.VelocitySolver(g, eta=_t(case["k"]), bc_cmb=bc[0], bc_surface=bc[1], gca=1, coarse_solver=T.COARSE_DENSE)
    fcells, fbytes = full.level_storage(1)
    assert fcells == int(np.prod(case["shells"][1].cell_shape)) and bytes1 < fbytes
    inv = s.inverse_diagonal(1)
    d = np.stack([t.cpu().numpy() for t in inv])
    assert rel_err(1.0 / d, golden[f"diag_{bc[0]}{bc[1]}_l1"]) < 1e-12
    # one FP64 V-cycle against the oracle's with the same (exact) coarsest solve
    lambdas = [None] + [s.level_lambda(l) for l in range(1, nlev)]
    o = s.options
    Hl = O.VelocityHierarchy(case["shell"], case["k"], bc[0], bc[1], nlev, gca=2, lambdas=lambdas,
                             cheb_order=o.chebyshev_order, cheb_iters=o.chebyshev_iterations, coarse_rtol=1e-14,
                             coarse_max_iter=5000)
    sh = case["shell"]
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 77)), *bc)
    ref = Hl.multigrid().solve(np.zeros(sh.vec_shape), b)
    x = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    s.vcycle(x, _t(b))
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    assert g.check_device_error() == 0


@pytest.mark.parametrize("bc", BC_L3)
def test_operator_api_matches_reference(cuda, golden, case, bc):
    """set_selective_matrices + gca_build level by level (TwoGridGCA on a Selective coarse operator), applied in
    Replace mode with the interface sum: the reference's coarse-operator applies and diagonals."""
    import torch

    lat, nlev = case["level"], case["num_levels"]
    g = T.Shell(lat, num_levels=nlev)
    marks = T.gca_mark_elements(g, nlev - 1, nlev - 1, _t(case["k"]))
    fine = T.EpsDivDiv(g, nlev - 1, k=_t(case["k"]), bc_cmb=0, bc_surface=0)
    ops = {}
    for l in range(nlev - 2, -1, -1):
        op = T.EpsDivDiv(g, l, k=_t(case["k_levels"][l]), bc_cmb=bc[0], bc_surface=bc[1])
        op.set_selective_matrices(l, marks)
        T.gca_build(fine if l == nlev - 2 else ops[l + 1], op)
        ops[l] = op
    for l in range(nlev - 1):
        u = _t(case["u"][l])
        out = torch.full_like(u, float("nan"))
        ops[l].apply(u, out)
        assert rel_err(out.cpu().numpy(), golden[f"apply_{bc[0]}{bc[1]}_l{l}"]) < 1e-12
        ops[l].set_diagonal(True)
        ops[l].apply(torch.ones_like(u), out)
        ops[l].set_diagonal(False)
        assert rel_err(out.cpu().numpy(), golden[f"diag_{bc[0]}{bc[1]}_l{l}"]) < 1e-12
    n, nbytes = ops[0].stored_cells()
    assert n == int(marks.sum().item()) and nbytes > 0
    assert g.check_device_error() == 0


def test_stokes_fgmres_history_matches_reference(cuda, golden):
    import torch

    case = selective_case(SELECTIVE_FGMRES)
    assert abs(checksum(case["k"]) - float(golden["fgmres_in_k"])) <= 1e-12 * abs(float(golden["fgmres_in_k"]))
    lat, nlev, bc = case["level"], case["num_levels"], case["bcs"]
    sh, shp = case["shell"], case["shell"].coarser()
    g = T.Shell(lat, num_levels=nlev)
    s = T.StokesSolver(g, eta=_t(case["k"]), bc_cmb=bc[0], bc_surface=bc[1], gca=2, relative_tolerance=1e-8,
                       absolute_tolerance=0.0, max_iterations=case["max_it"], normalize_pressure=0,
                       project_pressure_mean=0)
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [_t(case["f"][i]) for i in range(3)] + [torch.zeros_like(x[3])]
    s.solve(x, b)
    hist = np.array(s.history())
    want = golden["fgmres_history"]
    assert len(hist) == len(want)
    assert np.allclose(hist, want, rtol=1e-5, atol=0.0)
    marks = O.gca_marks(case["shell"], case["k"], nlev - 1)
    assert 0 < marks.sum() < marks.size
    assert s.level_storage(1)[0] == int(O.expand_marks(marks, 1).sum())


@pytest.mark.parametrize("interpolation", [T.TRANSFER_CONSTANT, T.TRANSFER_LINEAR])
def test_fast_build_equals_scalar_build(cuda, interpolation):
    """Three levels: level 3 from the on-the-fly level-4 matrices (rank form), level 2 from the stored level-3
    matrices (tensor-core triple products), both against the plain scalar build and the oracle."""
    sh = O.Shell(4)
    k = smooth_viscosity(sh, 57, 1000.0)
    g = T.Shell(4, num_levels=3)
    out = {}
    for tc in (True, False):
        fine = T.EpsDivDiv(g, 2, k=_t(k), bc_cmb=0, bc_surface=0)
        mid = T.EpsDivDiv(g, 1, k=_t(O.inject(sh.coarser(), k)), bc_cmb=0, bc_surface=0)
        nl0, nr0 = g.dims(0)
        coarse = T.EpsDivDiv(g, 0, k=_t(np.ones((10, nl0, nl0, nr0))), bc_cmb=0, bc_surface=0)
        T.gca_build(fine, mid, interpolation=interpolation, tensor_cores=tc)
        T.gca_build(mid, coarse, interpolation=interpolation, tensor_cores=tc)
        out[tc] = (mid.local_matrices(), coarse.local_matrices())
    assert rel_err(out[True][0], out[False][0]) < 1e-13
    assert rel_err(out[True][1], out[False][1]) < 1e-13
    lin = interpolation == T.TRANSFER_LINEAR
    m3 = O.gca_coarsen(O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN), linear=lin)
    sh3 = sh.coarser()
    m2 = O.gca_coarsen(O.EpsDivDiv(sh3, k=np.ones(sh3.scalar_shape), stored=m3), fine_mats=m3, linear=lin)
    assert rel_err(out[True][0], m3) < 1e-12
    assert rel_err(out[True][1], m2) < 1e-12


@pytest.mark.parametrize("gca", [1, 2])
def test_fp32_vcycle_freeslip_both(cuda, case, gca):
    """Free slip on both boundaries puts the null-space penalty into every level's apply; the FP32 V-cycle over
    FP64-built Galerkin levels uses the FP32 copy of the rotation modes and stays close to the FP64 V-cycle."""
    import torch

    lat, nlev = case["level"], case["num_levels"]
    sh = case["shell"]
    g = T.Shell(lat, num_levels=nlev)
    kw = dict(eta=_t(case["k"]), bc_cmb=2, bc_surface=2, gca=gca, coarse_solver=T.COARSE_DENSE)
    s64 = T.VelocitySolver(g, **kw)
    s32 = T.VelocitySolver(g, mixed_precision=1, **kw)
    b = O.enforce_rhs_bcs(sh, consistent(sh, O.seeded_normal(sh.vec_shape, 78)), 2, 2)
    x64 = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    s64.vcycle(x64, _t(b))
    x32 = torch.zeros(sh.vec_shape, dtype=torch.float32, device=cuda)
    s32.vcycle(x32, _t(b, torch.float32))
    assert rel_err(x32.double().cpu().numpy(), x64.cpu().numpy()) < 1e-4
    assert g.check_device_error() == 0
