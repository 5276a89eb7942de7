"""Mesh: the product's host generator against the oracle (bit-exact), plus the
reference's own known answers (tests/test_flag_field_unique_vertices.cpp)."""
import numpy as np
import pytest

import oracle as O
import terra_b200 as T


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4, 5, 6])
def test_product_mesh_bit_exact_vs_oracle(level):
    rad = max(level, 1)
    coords, radii, owned, cls, nc = T.mesh_generate_host(level, rad)
    sh = O.Shell(level, rad)
    assert np.array_equal(coords, sh.coords)  # bit-exact
    assert np.array_equal(radii, sh.radii)
    assert np.array_equal(owned, sh.owned_lat)
    assert nc == sh.num_classes

    def groups(c):
        g = {}
        for i, k in enumerate(c.reshape(-1)):
            if k >= 0:
                g.setdefault(int(k), []).append(i)
        return sorted(tuple(v) for v in g.values())

    assert groups(cls) == groups(sh.classes)


@pytest.mark.parametrize("level", [1, 2, 3, 4, 5])
def test_unique_node_counts(level):
    """Owned nodes == unique nodes; every duplicate class has exactly one owner
    (test_flag_field_unique_vertices.cpp:52-87)."""
    sh = O.Shell(level)
    n = sh.nl - 1
    owned = int(sh.owned.sum())
    assert owned == (10 * n * n + 2) * sh.nr
    # "additive communication of the mask": summing the ownership flag over each
    # class gives 1 everywhere
    flag = sh.owned.astype(np.float64)
    summed = sh.interface_sum(flag)
    assert summed.min() == 1.0 and summed.max() == 1.0
    assert summed.sum() == 10 * sh.nl * sh.nl * sh.nr


@pytest.mark.parametrize("level", [2, 4])
def test_mesh_geometry(level):
    sh = O.Shell(level)
    norms = np.linalg.norm(sh.coords, axis=-1)
    assert np.abs(norms - 1.0).max() < 1e-15
    cls = sh.classes.reshape(-1)
    c = sh.coords.reshape(-1, 3)
    sizes = np.bincount(cls[cls >= 0])
    # 12 base vertices: poles shared by 5 diamonds, ring vertices by 3; edge nodes by 2
    assert sorted(set(sizes.tolist())) == [2, 3, 5]
    assert (sizes == 5).sum() == 2 and (sizes == 3).sum() == 10
    for k in range(sh.num_classes):
        m = np.where(cls == k)[0]
        assert np.all(c[m] == c[m[0]])  # duplicates are the same point, bit for bit
    # radii: uniform, r_max exact (spherical_shell.hpp:27-52)
    assert sh.radii[0] == 0.55 and sh.radii[-1] == 1.0
    assert np.allclose(np.diff(sh.radii), 0.45 / (sh.nr - 1))


def test_boundary_flags():
    sh = O.Shell(2)
    m = sh.boundary_mask
    assert np.all(m[..., 0] == 6) and np.all(m[..., -1] == 10) and np.all(m[..., 1:-1] == 1)
