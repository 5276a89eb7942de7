"""Adaptive GCA (gca = 2) in the oracle, against the reference.

GCAElementsCollector (gca_elements_collector.hpp:49-103) marks coarsest cells where a fine wedge's coefficient
gradient in reference coordinates exceeds 10; the coarse operators then store Galerkin matrices on the
descendants of marked cells only and re-discretise elsewhere (OperatorStoredMatrixMode::Selective,
local_matrix_storage.hpp:22-166, the slow path's per-cell choice epsilon_divdiv_kerngen.hpp:1047-1060). The
fixture tests/golden/ref_gca_selective.npz holds the reference's marks, coarse-operator applies and diagonals
of a level-4 hierarchy; the oracle must reproduce the marks exactly and the applies to 1e-12.
"""
import os

import numpy as np
import pytest

import oracle as O
import ref as R
from golden_inputs import BC_L3, MARK_CASES, checksum, selective_case
from helpers import rel_err, smooth_viscosity

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_gca_selective.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", MARK_CASES)
def test_oracle_marks_equal_reference(golden, case):
    lat, lr, seed, contrast = case
    sh = O.Shell(lat)
    m = O.gca_marks(sh, smooth_viscosity(sh, seed, contrast), lr)
    want = golden[f"marks_L{lat}_r{lr}_s{seed}"].astype(bool)
    assert 0 < want.sum() < want.size  # the case marks some cells, not all
    assert np.array_equal(m, want)


def test_expand_marks_follows_map_to_coarse_element():
    marks = np.zeros((10, 2, 2, 2), bool)
    marks[3, 1, 0, 1] = True
    e = O.expand_marks(marks, 2)
    d, x, y, r = np.nonzero(e)
    assert len(d) == 64 and set(d) == {3}
    assert set(x >> 2) == {1} and set(y >> 2) == {0} and set(r >> 2) == {1}


@pytest.fixture(scope="module")
def case():
    return selective_case()


@pytest.mark.parametrize("bc", BC_L3)
def test_oracle_selective_hierarchy_matches_reference(golden, case, bc):
    assert abs(checksum(case["k"]) - float(golden["in_k"])) <= 1e-12 * abs(float(golden["in_k"]))
    nlev = case["num_levels"]
    H = O.VelocityHierarchy(case["shell"], case["k"], bc[0], bc[1], nlev, gca=2, lambdas=[None] + [1.0] * (nlev - 1))
    assert 0 < H.marks.sum() < H.marks.size
    for l in range(nlev - 1):
        u = case["u"][l]
        assert rel_err(H.ops[l].apply(u), golden[f"apply_{bc[0]}{bc[1]}_l{l}"]) < 1e-12
        assert rel_err(H.ops[l].apply(np.ones_like(u), diagonal=True), golden[f"diag_{bc[0]}{bc[1]}_l{l}"]) < 1e-12


def test_selective_differs_from_full_and_rediscretised(case):
    """The case exercises both kinds of cell: the adaptive operator is neither the Galerkin nor the rediscretised
    one."""
    nlev, lam = case["num_levels"], [None] + [1.0] * (case["num_levels"] - 1)
    sel, full, redisc = (O.VelocityHierarchy(case["shell"], case["k"], 1, 1, nlev, gca=g, lambdas=lam)
                         for g in (2, 1, 0))
    u = case["u"][0]
    a = sel.ops[0].apply(u)
    assert rel_err(a, full.ops[0].apply(u)) > 1e-3
    assert rel_err(a, redisc.ops[0].apply(u)) > 1e-2


@pytest.mark.skipif(not R.available(), reason="compiled reference (oracle/_ref) not present")
def test_oracle_marks_equal_live_reference():
    sh = O.Shell(4)
    k = smooth_viscosity(sh, 21, 3e4)
    m = O.gca_marks(sh, k, 2)
    assert 0 < m.sum() < m.size
    assert np.array_equal(m, R.gca_marks(4, 2, k))
