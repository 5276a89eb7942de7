"""The CUDA path against outputs of the reference itself, through the C ABI.

Fixtures (tests/golden/, written by tests/golden/make_golden.py from the reference's own FP64 code): every
operator apply, B, B^T, the masses, the transfers and the Galerkin element matrices within 1e-12 relative
(max norm), the right-hand-side boundary treatment within 1e-13, and the Stokes FGMRES residual history step
by step within 1e-5 relative. Where the compiled reference (oracle/_ref/) travelled with the repository, the
level-6 benchmark configuration (spherical-harmonic viscosity, no-slip CMB, free-slip surface) is also
compared live: the fine-level apply, B and B^T at 1e-12, and the first five FGMRES residuals of the
unprojected solve at 1e-6.
"""
import os

import numpy as np
import pytest

import oracle as O
import ref as R
import terra_b200 as T
from golden_inputs import BC_ALL, BC_L3, FGMRES_CASES, checksum, level_inputs, stokes_case
from helpers import rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL64 = 1e-12


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def _t(a, cuda):
    import torch

    return torch.tensor(np.ascontiguousarray(a), device=cuda)


def _np(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("lat,bcs_list", [(2, BC_ALL), (3, BC_L3)])
def test_operators_match_reference(cuda, lat, bcs_list):
    import torch

    g = _load(f"ref_ops_L{lat}.npz")
    inp = level_inputs(lat)
    assert abs(checksum(inp["u"]) - float(g["in_u"])) <= 1e-12 * abs(float(g["in_u"]))
    sh, k, u, p = inp["shell"], inp["k"], inp["u"], inp["p"]
    gs = T.Shell(lat, num_levels=2)
    kk, uu, pp = _t(k, cuda), _t(u, cuda), _t(p, cuda)
    for bc in bcs_list:
        tag = f"{bc[0]}{bc[1]}"
        A = T.EpsDivDiv(gs, 1, k=kk, bc_cmb=bc[0], bc_surface=bc[1])
        out = torch.full_like(uu, float("nan"))
        A.apply(uu, out)
        assert rel_err(_np(out), g[f"apply_fast_{tag}"]) < TOL64, tag
        Ad = T.EpsDivDiv(gs, 1, k=kk, bc_cmb=bc[0], bc_surface=bc[1], diagonal=True)
        Ad.apply(torch.ones_like(uu), out)
        assert rel_err(_np(out), g[f"diag_{tag}"]) < TOL64, tag
        if lat == 2:
            A.set_modes(T.REPLACE, T.SKIP_COMMUNICATION)
            A.apply(uu, out)
            assert rel_err(_np(out), g[f"apply_skipcomm_{tag}"]) < TOL64, tag
        B = T.Divergence(gs, 1, bc_cmb=bc[0], bc_surface=bc[1])
        BT = T.Gradient(gs, 1, bc_cmb=bc[0], bc_surface=bc[1])
        po = torch.full_like(pp, float("nan"))
        B.apply(uu, po)
        assert rel_err(_np(po), g[f"div_{tag}"]) < TOL64, tag
        BT.apply(pp, out)
        assert rel_err(_np(out), g[f"grad_{tag}"]) < TOL64, tag
    Aq = T.EpsDivDiv(gs, 1, k_cell=_t(inp["k_q0"], cuda), bc_cmb=1, bc_surface=2)
    out = torch.zeros_like(uu)
    Aq.apply(uu, out)
    assert rel_err(_np(out), g["apply_q0_12"]) < TOL64
    d = torch.zeros_like(kk)
    T.kmass_lumped_diagonal(gs, 1, kk, d)
    assert rel_err(_np(d), g["kmass"]) < TOL64
    T.vector_mass_apply(gs, 1, uu, out)
    assert rel_err(_np(out), g["vmass"]) < TOL64
    fine = uu.clone()
    T.prolongate_add(gs, 1, _t(inp["u_coarse"], cuda), fine)
    assert rel_err(_np(fine), g["prolong_add"]) < TOL64
    coarse = torch.zeros((3,) + sh.coarser().scalar_shape, dtype=torch.float64, device=cuda)
    T.restrict(gs, 1, uu, coarse)
    assert rel_err(_np(coarse), g["restrict"]) < TOL64
    assert gs.check_device_error() == 0


def test_gca_and_rhs_match_reference(cuda):
    g = _load("ref_ops_L3.npz")
    inp = level_inputs(3)
    gs = T.Shell(3, num_levels=2)
    fine = T.EpsDivDiv(gs, 1, k=_t(inp["k"], cuda), bc_cmb=0, bc_surface=0)
    nc = inp["shell"].coarser().nl
    coarse = T.EpsDivDiv(gs, 0, k=_t(np.ones((10, nc, nc, nc)), cuda), bc_cmb=0, bc_surface=0)
    T.gca_build(fine, coarse)
    m = coarse.local_matrices()
    assert rel_err(m[0], g["gca_d0"]) < TOL64
    assert abs((m * m).sum() - g["gca_sumsq"][0]) <= 1e-12 * g["gca_sumsq"][0]
    T.gca_build(fine, coarse, interpolation=T.TRANSFER_LINEAR)
    assert rel_err(coarse.local_matrices()[0], g["gca_linear_d0"]) < TOL64
    import torch

    uu = _t(inp["u"], cuda)
    fine_v = uu.clone()
    T.prolongate_linear_add(gs, 1, _t(inp["u_coarse"], cuda), fine_v)
    assert rel_err(_np(fine_v), g["prolong_linear_add"]) < TOL64
    cv = torch.zeros((3,) + inp["shell"].coarser().scalar_shape, dtype=torch.float64, device=cuda)
    T.restrict_linear(gs, 1, uu, cv)
    assert rel_err(_np(cv), g["restrict_linear"]) < TOL64
    u = inp["u"]
    for bc in ((1, 2), (2, 1), (1, 1)):
        v = _t(u, cuda)
        T.stokes_rhs_enforce(gs, 1, v, bc[0], bc[1])
        assert rel_err(_np(v).ravel(), g[f"rhs_{bc[0]}{bc[1]}"][: u.size]) < 1e-13


@pytest.mark.parametrize("name", list(FGMRES_CASES))
def test_stokes_fgmres_matches_reference(cuda, name):
    import torch

    g = _load("ref_fgmres_L3.npz")
    c = stokes_case(**FGMRES_CASES[name])
    sh, shp = c["shell"], c["shell"].coarser()
    gs = T.Shell(c["level"], num_levels=c["num_levels"])
    solver = T.StokesSolver(gs, eta=_t(c["k"], cuda), bc_cmb=c["bcs"][0], bc_surface=c["bcs"][1], gca=1,
                            relative_tolerance=c["rtol"], absolute_tolerance=0.0, max_iterations=c["max_it"],
                            normalize_pressure=0, project_pressure_mean=0)
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [_t(c["f"][i], cuda) for i in range(3)] + [torch.zeros_like(x[3])]
    solver.solve(x, b)
    hist = np.array(solver.history())
    want = g[f"{name}_history"]
    assert len(hist) == len(want)
    assert np.allclose(hist[:31], want[:31], rtol=1e-5, atol=0.0)
    if name == "noslip":
        assert np.allclose(hist, want, rtol=1e-5, atol=0.0)
        xr = g[f"{name}_x"]
        nu = 3 * int(np.prod(sh.scalar_shape))
        ug = np.concatenate([_np(t).ravel() for t in x[:3]])
        assert rel_err(ug, xr[:nu]) < 1e-7
        pg, pr = _np(x[3]).ravel(), xr[nu:]
        own = shp.owned.ravel()
        assert rel_err(pg - pg[own].mean(), pr - pr[own].mean()) < 1e-7
    else:
        # stagnation near the unprojected floor amplifies rounding differences
        assert np.allclose(hist, want, rtol=1e-4, atol=0.0)


needs_ref = pytest.mark.skipif(not R.available(), reason="compiled reference (oracle/_ref) not present")


class _HostShell:
    def __init__(self, sh):
        self.sh = sh

    def coords(self, level):
        return self.sh.coords

    def radii(self, level):
        return self.sh.radii


@needs_ref
def test_level6_benchmark_configuration_matches_live_reference(cuda):
    """The level-6 benchmark configuration against the reference itself: fine-level apply, B, B^T, and the first
    five FGMRES residuals of the FP64 solve without the pressure-mean projection."""
    import torch

    import synthetic as S

    lat, nlev, bcs = 6, 5, (1, 2)
    sh = O.Shell(lat)
    shp = sh.coarser()
    eta = S.viscosity(_HostShell(sh), 0, seed=1)
    u = O.seeded_normal(sh.vec_shape, 61)
    gs = T.Shell(lat, num_levels=nlev)
    ee, uu = _t(eta, cuda), _t(u, cuda)
    A = T.EpsDivDiv(gs, nlev - 1, k=ee, bc_cmb=bcs[0], bc_surface=bcs[1])
    out = torch.zeros_like(uu)
    A.apply(uu, out)
    assert rel_err(_np(out), R.epsdivdiv(lat, u, k=eta, bc_cmb=bcs[0], bc_surface=bcs[1])) < TOL64
    B = T.Divergence(gs, nlev - 1, bc_cmb=bcs[0], bc_surface=bcs[1])
    po = torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda)
    B.apply(uu, po)
    assert rel_err(_np(po), R.divergence(lat, u, *bcs)) < TOL64
    p = O.seeded_normal(shp.scalar_shape, 62)
    T.Gradient(gs, nlev - 1, bc_cmb=bcs[0], bc_surface=bcs[1]).apply(_t(p, cuda), out)
    assert rel_err(_np(out), R.gradient(lat, p, *bcs)) < TOL64

    # right-hand side of the benchmark kind, assembled by the reference itself
    rng = np.random.default_rng(63)
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    Tf = np.cos(X @ rng.normal(size=3) * 2.0)
    f = R.vector_mass(lat, np.moveaxis(Tf[..., None] * rhat, -1, 0))
    b = R.rhs_enforce(lat, np.concatenate([f.ravel(), np.zeros(shp.scalar_shape).ravel()]), *bcs)
    shells = [sh]
    for _ in range(nlev - 1):
        shells.insert(0, shells[0].coarser())
    starts = [O.seeded_uniform(shells[l], 3, 12345 + 7919 * l) for l in range(nlev)]
    ref = R.StokesRef(lat, nlev, eta, 1.0 / O.inject(shp, eta), start=starts, bc_cmb=bcs[0], bc_surface=bcs[1])
    _, want, _ = ref.solve(b, rtol=1e-8, atol=0.0, max_it=5)
    ref.close()

    solver = T.StokesSolver(gs, eta=ee, bc_cmb=bcs[0], bc_surface=bcs[1], gca=1, relative_tolerance=1e-8,
                            absolute_tolerance=0.0, max_iterations=5, normalize_pressure=0, project_pressure_mean=0)
    nu = 3 * int(np.prod(sh.scalar_shape))
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    bu = b[:nu].reshape(sh.vec_shape)
    bb = [_t(bu[i], cuda) for i in range(3)] + [_t(b[nu:].reshape(shp.scalar_shape), cuda)]
    solver.solve(x, bb)
    hist = np.array(solver.history())
    assert len(hist) == len(want) == 6
    assert np.allclose(hist, want, rtol=1e-6, atol=0.0)
