"""The reference's manufactured Stokes solution (tests/test_epsilon_divdiv_
stokes.cpp:93-238; set-up in tests/test_manufactured.py) solved by the product:
at level 4 its discretisation errors equal the oracle's (both solves to
1e-10), and from level 4 to level 5 they fall at second order, in FP64 and
with the FP32 V-cycle."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from test_manufactured import _solve as oracle_solve
from test_manufactured import manufactured_system, owned_l2_errors

pytestmark = pytest.mark.gpu


def _product_errors(level, mixed, cuda):
    import torch

    sh, shp, k, u_ex, p_ex, bu, bp = manufactured_system(level)
    g = T.Shell(level, num_levels=level)
    solver = T.StokesSolver(g, eta=torch.tensor(k, device=cuda), bc_cmb=T.DIRICHLET, bc_surface=T.DIRICHLET,
                            relative_tolerance=1e-10, absolute_tolerance=0.0, max_iterations=600, restart=64,
                            mixed_precision=mixed, project_pressure_mean=0, normalize_pressure=0)
    x = [torch.zeros(sh.scalar_shape, dtype=torch.float64, device=cuda) for _ in range(3)]
    x.append(torch.zeros(shp.scalar_shape, dtype=torch.float64, device=cuda))
    b = [torch.tensor(np.ascontiguousarray(bu[c]), device=cuda) for c in range(3)]
    b.append(torch.tensor(np.ascontiguousarray(bp), device=cuda))
    assert solver.solve(x, b)
    u = np.stack([x[c].cpu().numpy() for c in range(3)])
    return owned_l2_errors(sh, shp, u, x[3].cpu().numpy(), u_ex, p_ex)


@pytest.mark.parametrize("mixed", [0, 1])
def test_manufactured_solution_product(cuda, mixed):
    (eu_o, ep_o), _ = oracle_solve(4)
    eu4, ep4 = _product_errors(4, mixed, cuda)
    assert abs(eu4 - eu_o) <= 1e-6 * eu_o
    assert abs(ep4 - ep_o) <= 1e-6 * ep_o
    eu5, ep5 = _product_errors(5, mixed, cuda)
    assert 3.5 < eu4 / eu5 < 4.5
    assert 3.0 < ep4 / ep5 < 4.5
