"""The flat-grid kernels (B, B^T, transfers) decode a thread index with
q = (i * (floor(2^40 / n) + 1)) >> 40 in 64-bit unsigned arithmetic (Decoder
in tn_kernels.hpp). Check, exhaustively on the CPU, that this equals i // n
and that the product stays below 2^64 for every divisor and index range the
kernels use on levels 0..7 (radial entries nr or nr - 1, lateral nl or
nl - 1, fine and coarse)."""
import numpy as np


def _recip(n):
    return (1 << 40) // n + 1


def _check(n, count):
    m = _recip(n)
    assert (count - 1) * m < 1 << 64
    i = np.arange(count, dtype=np.uint64)
    q = (i * np.uint64(m)) >> np.uint64(40)
    assert np.array_equal(q, i // np.uint64(n)), (n, count)


def test_decoder_exact_on_all_levels():
    for level in range(0, 8):
        nl = (1 << level) + 1
        nr = nl
        for lat, rad in ((nl, nr), (nl - 1, nr - 1)):  # nodes, cells
            if lat < 1 or rad < 1:
                continue
            entries = 10 * lat * lat * rad
            _check(rad, entries)  # i -> lateral column
            _check(lat, 10 * lat * lat)  # column -> (d * lat + x)
            _check(lat, 10 * lat)  # (d * lat + x) -> d


def test_decoder_bound_for_mixed_radial_levels():
    """Shells with a different radial level (e.g. 9 x 9 x 129): the decode is
    exact for i < 2^40 / n and the 64-bit product cannot overflow for every
    divisor n <= 129 and index below 10 * 129^2 * 129."""
    imax = 10 * 129 * 129 * 129
    for n in range(1, 130):
        m = _recip(n)
        assert imax < (1 << 40) // n
        if n >= 2:
            assert imax * m < 1 << 64
    # n = 1 occurs only at level 0 (2 x 2 lateral nodes), where indices stay tiny
    assert 10 * 2 * 2 * 129 * _recip(1) < 1 << 64
