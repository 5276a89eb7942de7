"""GPU checks of the VectorLike operations and the right-hand-side boundary kernels of the C ABI against the
oracle (numpy restatements of grid_operations.hpp and local_basis_trafo_normal_tangential.hpp)."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import consistent, rel_err

pytestmark = pytest.mark.gpu


def _setup(cuda, level=3, seed=3):
    import torch

    sh = O.Shell(level)
    g = T.Shell(level)
    a = O.seeded_normal(sh.vec_shape, seed)
    return sh, g, a, torch.tensor(a, device=cuda)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_invert_scale_swap_max_abs(cuda, dtype):
    import torch

    sh, g, a, t = _setup(cuda)
    dt = torch.float64 if dtype == "f64" else torch.float32
    tol = 1e-15 if dtype == "f64" else 1e-6
    y = t.to(dt).clone()
    T.vec_invert(g, 0, y)
    assert rel_err(y.double().cpu().numpy(), 1.0 / a.astype(np.float32 if dtype == "f32" else np.float64)) < tol
    x = torch.tensor(O.seeded_normal(sh.vec_shape, 4), device=cuda, dtype=dt)
    y = t.to(dt).clone()
    T.vec_scale(g, 0, y, x)
    assert rel_err(y.double().cpu().numpy(), (t.to(dt) * x).double().cpu().numpy()) == 0.0
    y0, x0 = t.to(dt).clone(), x.clone()
    T.vec_swap(g, 0, y0, x0)
    assert torch.equal(y0, x) and torch.equal(x0, t.to(dt))
    assert T.vec_max_abs(g, 0, t.to(dt)) == float(t.to(dt).abs().max())
    assert not T.vec_has_nan_or_inf(g, 0, t.to(dt))


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_has_nan_or_inf(cuda, bad):
    """NaN / Inf placed in host-prepared input is reported (grid_operations.hpp:331-346)."""
    sh, g, a, t = _setup(cuda)
    t[1, 3, 2, 1, 4] = bad
    assert T.vec_has_nan_or_inf(g, 0, t)
    assert T.vec_has_nan_or_inf(g, 0, [t[1]])
    assert not T.vec_has_nan_or_inf(g, 0, [t[0]])


def test_cast_roundtrip(cuda):
    import torch

    _, _, a, t = _setup(cuda)
    f = torch.empty(t.shape, dtype=torch.float32, device=cuda)
    T.vec_cast(t, f)
    assert torch.equal(f, t.float())
    back = torch.empty_like(t)
    T.vec_cast(f, back)
    assert torch.equal(back, f.double())


@pytest.mark.parametrize("flag", [T.FLAG_CMB, T.FLAG_SURFACE, T.FLAG_BOUNDARY, T.FLAG_INNER, 0])
def test_assign_masked_and_freeslip(cuda, flag):
    sh, g, a, t = _setup(cuda)
    v = t.clone()
    T.vec_assign_masked(g, 0, v, flag, 2.5)
    assert rel_err(v.cpu().numpy(), O.assign_masked(sh, a, flag, 2.5)) == 0.0
    v = t.clone()
    T.vec_freeslip_project(g, 0, v, flag)
    assert rel_err(v.cpu().numpy(), O.freeslip_project(sh, a, flag)) < 1e-14
    v = t.clone()
    T.vec_rotate_normal_tangential(g, 0, v, flag, 0)
    T.vec_rotate_normal_tangential(g, 0, v, flag, 1)
    assert rel_err(v.cpu().numpy(), a) < 1e-15


@pytest.mark.parametrize("bcs", [(1, 2), (2, 1), (1, 1), (2, 2), (0, 1)])
def test_stokes_rhs_enforce_matches_oracle(cuda, bcs):
    sh, g, a, t = _setup(cuda)
    a = consistent(sh, a)
    import torch

    v = torch.tensor(a, device=cuda)
    T.stokes_rhs_enforce(g, 0, v, *bcs)
    assert rel_err(v.cpu().numpy(), O.rhs_enforce_app(sh, a, *bcs)) < 1e-14


def test_freeslip_penalty_matches_oracle(cuda):
    """Free slip on both boundaries: the apply carries the reference's 1e-7 rotation penalty; on a rigid
    rotation (in the operator's null space) the output is the penalty alone."""
    import torch

    level = 3
    sh = O.Shell(level)
    k = np.exp(np.sin(sh.physical_coords() @ np.array([1.0, 2.0, -1.0])))
    X = sh.physical_coords()
    w = np.array([0.3, -0.7, 0.5])
    rot = np.moveaxis(np.cross(w, X), -1, 0).copy()
    g = T.Shell(level)
    op = T.EpsDivDiv(g, 0, k=torch.tensor(k, device=cuda), bc_cmb=2, bc_surface=2)
    out = torch.zeros(sh.vec_shape, dtype=torch.float64, device=cuda)
    op.apply(torch.tensor(rot, device=cuda), out)
    ref = O.EpsDivDiv(sh, k=k, bc_cmb=2, bc_surface=2).apply(rot)
    plain = O.EpsDivDiv(sh, k=k, bc_cmb=2, bc_surface=1).apply(consistent(sh, O.seeded_normal(sh.vec_shape, 9)))
    # the penalty (about 1e-7 of the input) dominates; rounding of A rot is ~1e-15 of a generic apply
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-13 * np.abs(plain).max()
    assert np.abs(ref).max() > 1e3 * 1e-15 * np.abs(plain).max()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_vec_alloc_free_and_sync(cuda, dtype):
    """tn_vec_alloc gives zero-filled, 256-byte-aligned arrays of the level's nodes that the other entry points
    accept; seeded values written into them read back through tn_vec_max_abs; tn_sync returns TN_OK."""
    import ctypes

    import torch

    dt = torch.float64 if dtype == "f64" else torch.float32
    g = T.Shell(3, num_levels=2)
    v = T.DeviceVector(g, 1, 3, dt)
    assert all(p % 256 == 0 for p in v.pointers)
    L = T.load()
    prec = T.TN_F64 if dtype == "f64" else T.TN_F32
    arr = (ctypes.c_void_p * 3)(*v.pointers)
    out = ctypes.c_double()
    assert L.tn_vec_max_abs(g.handle, 1, prec, 3, arr, ctypes.byref(out), None) == 0
    assert out.value == 0.0
    assert L.tn_vec_random(g.handle, 1, prec, 3, ctypes.c_uint64(7), arr, None) == 0
    T.sync()
    assert L.tn_vec_max_abs(g.handle, 1, prec, 3, arr, ctypes.byref(out), None) == 0
    assert 0.5 < out.value <= 1.0  # uniform(-1, 1) over 3 x 10 x 9 x 9 x 9 values
    del v
    T.sync()
