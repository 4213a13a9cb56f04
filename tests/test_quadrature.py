"""Level-symmetric S_N sets: counts, quadrant order, weights, moment exactness."""
import math

import numpy as np
import pytest

from idcsweep.quadrature import SN_COUNTS_2D, level_symmetric_2d, level_symmetric_octant, moment_errors


@pytest.mark.parametrize("N", [2, 4, 6, 8, 12, 16])
def test_counts_order_and_weights(N):
    xi, eta, w, qb = level_symmetric_2d(N)
    assert xi.size == SN_COUNTS_2D[N]
    assert list(qb) == [0, xi.size // 4, xi.size // 2, 3 * xi.size // 4, xi.size]
    assert abs(w.sum() - 4 * math.pi) < 1e-12
    assert (w > 0).all()
    assert np.all(xi * xi + eta * eta < 1.0)
    for k in range(4):
        s = slice(qb[k], qb[k + 1])
        assert np.all(np.sign(xi[s]) == (-1 if k >= 2 else 1))
        assert np.all(np.sign(eta[s]) == (-1 if k & 1 else 1))
        # decreasing (xi, eta) inside the quadrant, OrdinateData::Compare order
        pairs = list(zip(xi[s], eta[s]))
        assert pairs == sorted(pairs, reverse=True)


@pytest.mark.parametrize("N,mu1", [(4, 0.3500212), (8, 0.2182179), (12, 0.1672127)])
def test_lq_n_sets_are_exact(N, mu1):
    m, _, _ = level_symmetric_octant(N)
    assert abs(m - mu1) < 5e-8
    err = moment_errors(N)
    pure = max(abs(err[(a, 0, 0)]) for a in range(N // 2 + 1))
    assert pure < 1e-13


def test_s16_moments_close():
    err = moment_errors(16)
    assert max(abs(v) for v in err.values()) < 1e-8
