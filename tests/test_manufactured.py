"""The reference's manufactured Stokes solution as a known-answer test of the
oracle (tests/test_epsilon_divdiv_stokes.cpp:93-238, 459-520): velocity
u = (-4 cos 4z, 8 cos 8x, -2 cos 2y), pressure p = sin 4x sin 8y sin 2z,
viscosity k = 2 + sin z, the matching right-hand side f, Dirichlet boundary
values lifted the reference's way (strong_algebraic_velocity_dirichlet_
enforcement_stokes_like: b -= K_neumann g, boundary rows = diag(K_neumann) g).

Solved with the oracle's FGMRES and block-triangular GMG preconditioner to
1e-10 on levels 2, 3, 4 (as in the reference's level loop), the owned-node L2
errors must fall at second order (ratio ~4 per level; observed 4.05 / 3.86 for
velocity, 3.44 / 4.13 for pressure) with a level-independent iteration count
(43-46)."""
import numpy as np

import oracle as O


def _exact(X):
    x, y, z = X[..., 0], X[..., 1], X[..., 2]
    u = np.stack([-4 * np.cos(4 * z), 8 * np.cos(8 * x), -2 * np.cos(2 * y)])
    p = np.sin(4 * x) * np.sin(8 * y) * np.sin(2 * z)
    f = np.stack([-64.0 * (np.sin(z) + 2) * np.cos(4 * z) - 16.0 * np.sin(4 * z) * np.cos(z)
                  + 4 * np.sin(8 * y) * np.sin(2 * z) * np.cos(4 * x),
                  512.0 * (np.sin(z) + 2) * np.cos(8 * x) + 8 * np.sin(4 * x) * np.sin(2 * z) * np.cos(8 * y)
                  - 4.0 * np.sin(2 * y) * np.cos(z),
                  -8.0 * (np.sin(z) + 2) * np.cos(2 * y) + 2 * np.sin(4 * x) * np.sin(8 * y) * np.cos(2 * z)])
    return u, p, f, 2.0 + np.sin(z)


def manufactured_system(level):
    """(shell, pressure shell, k, exact u, exact p, velocity rhs, pressure rhs)."""
    sh = O.Shell(level)
    shp = sh.coarser()
    u_ex, _, f_int, k = _exact(sh.physical_coords())
    _, p_ex, _, _ = _exact(shp.physical_coords())
    g = np.zeros_like(u_ex)
    g[..., 0], g[..., -1] = u_ex[..., 0], u_ex[..., -1]
    a_n = O.EpsDivDiv(sh, k=k, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN)
    b_n = O.Divergence(sh, bc_cmb=O.NEUMANN, bc_surface=O.NEUMANN)
    bu = O.vector_mass(sh, f_int) - a_n.apply(g)
    bp = -b_n.apply(g)
    dg = a_n.diag() * g
    bu[..., 0], bu[..., -1] = dg[..., 0], dg[..., -1]
    return sh, shp, k, u_ex, p_ex, bu, bp


def owned_l2_errors(sh, shp, u, p, u_ex, p_ex):
    own, ownp = sh.owned, shp.owned
    pm, pe = p - p[ownp].mean(), p_ex - p_ex[ownp].mean()
    eu = np.sqrt(np.sum((u - u_ex)[:, own] ** 2) / (3 * own.sum()))
    ep = np.sqrt(np.sum((pm - pe)[ownp] ** 2) / ownp.sum())
    return eu, ep


def _solve(level):
    sh, shp, k, u_ex, p_ex, bu, bp = manufactured_system(level)
    H = O.VelocityHierarchy(sh, k, O.DIRICHLET, O.DIRICHLET, level, gca=True, lambdas=[None] * level)
    H.lambdas = [None] + [H.power_iteration(l, O.seeded_uniform(H.shells[l], 3, 12345 + 7919 * l), 10)
                          for l in range(1, level)]
    St = O.StokesSystem(sh, k, O.DIRICHLET, O.DIRICHLET, H)
    b = St.join(bu, bp)
    hist = []
    x, its = O.fgmres(St.apply, np.zeros_like(b), b, St.dot, St.precondition, 100, 1e-10, 0.0, 600, hist)
    assert hist[-1] <= 1e-10
    u, p = St.split(x)
    return owned_l2_errors(sh, shp, u, p, u_ex, p_ex), its


def test_manufactured_solution_second_order():
    errs, its = zip(*[_solve(level) for level in (2, 3, 4)])
    for coarse, fine in zip(errs[:-1], errs[1:]):
        assert 3.5 < coarse[0] / fine[0] < 4.5  # velocity
        assert 3.0 < coarse[1] / fine[1] < 4.5  # pressure
    assert max(its) - min(its) <= 10
