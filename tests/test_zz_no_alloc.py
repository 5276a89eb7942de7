"""The static-scratch divergence entry point (tn_divergence_apply_noalloc):
the same result as the operator path on two calls in a row, no change in the
device's free memory or in torch's caching pool across the calls, and a clear error beyond its scratch
limit. Kept in the last-collected file so it also runs after every other test."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T
from helpers import consistent

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [3, 5])
@pytest.mark.parametrize("bcs", [(1, 1), (1, 2)])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_divergence_matches_operator(cuda, level, bcs, dtype):
    import torch

    dt = torch.float64 if dtype == "f64" else torch.float32
    sh = O.Shell(level)
    shp = sh.coarser()
    g = T.Shell(level, num_levels=2)
    B = T.Divergence(g, 1, dtype=dt, bc_cmb=bcs[0], bc_surface=bcs[1])
    # set-up call: looks up the scratch address (the driver may load the module here)
    warm = torch.zeros(sh.vec_shape, dtype=dt, device=cuda)
    T.divergence_apply_noalloc(g, 1, warm, torch.zeros(shp.scalar_shape, dtype=dt, device=cuda),
                               bc_cmb=bcs[0], bc_surface=bcs[1])
    for seed in (90, 91):  # two calls in a row, different inputs
        u = torch.tensor(consistent(sh, O.seeded_normal(sh.vec_shape, seed)), dtype=dt, device=cuda)
        ref = torch.full(shp.scalar_shape, float("nan"), dtype=dt, device=cuda)
        B.apply(u, ref)
        out = torch.full(shp.scalar_shape, float("nan"), dtype=dt, device=cuda)
        torch.cuda.synchronize()
        # torch's own pool first (an allocation it would serve without a new cudaMalloc), then the device's
        # free memory; the device figure may drift with other processes, so it is retried before failing
        alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
        for attempt in range(3):
            free0 = torch.cuda.mem_get_info()[0]
            T.divergence_apply_noalloc(g, 1, u, out, bc_cmb=bcs[0], bc_surface=bcs[1])
            torch.cuda.synchronize()
            if torch.cuda.mem_get_info()[0] == free0:
                break
        else:
            pytest.fail("device free memory changed across three calls")
        assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == reserved0
        a, b = out.double().cpu().numpy(), ref.double().cpu().numpy()
        tol = 1e-13 if dtype == "f64" else 1e-5
        assert np.abs(a - b).max() <= tol * np.abs(b).max()


def test_noalloc_divergence_rejects_levels_beyond_its_scratch(cuda):
    import torch

    g = T.Shell(6, num_levels=2)
    nl, nr = g.dims(1)
    nlc, nrc = g.dims(0)
    u = torch.zeros((3, 10, nl, nl, nr), dtype=torch.float64, device=cuda)
    p = torch.zeros((10, nlc, nlc, nrc), dtype=torch.float64, device=cuda)
    with pytest.raises(T.TerraError) as e:
        T.divergence_apply_noalloc(g, 1, u, p)
    assert e.value.code == -1 and "static scratch" in str(e.value)
