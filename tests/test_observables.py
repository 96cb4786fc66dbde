"""J-summed quantities over centrifugal-sudden blocks (qd_b200.observables)."""
import numpy as np
import pytest

from qd_b200.observables import k_averaged, integral_cross_section


def test_k_average_counts_each_projection():
    # j0 = 2: K = 0 once, K = 1, 2 twice, over 2 j0 + 1 = 5 projections
    E = np.linspace(0.01, 0.05, 7)
    blocks = {0: np.full(7, 0.5), 1: np.full(7, 0.2), 2: np.full(7, 0.1)}
    assert np.allclose(k_averaged(blocks, 10, 2), (0.5 + 2 * 0.2 + 2 * 0.1) / 5)
    # J = 1 admits only |K| <= 1
    assert np.allclose(k_averaged(blocks, 1, 2), (0.5 + 2 * 0.2) / 5)
    assert E.size == 7


def test_cross_section_known_answers():
    E = np.array([0.01, 0.02])
    mu = 1000.0
    # P_J = 1 for J = 0..Jmax: sigma = pi/k^2 (Jmax + 1)^2
    P = np.ones((21, 2))
    s = integral_cross_section(E, mu, P)
    assert np.allclose(s, np.pi / (2 * mu * E) * 21 ** 2)
    # P linear in J, given every 5: the interpolated sum is exact
    Js = np.arange(0, 21, 5)
    lin = lambda J: 0.9 - 0.04 * J
    s_sparse = integral_cross_section(E, mu, np.stack([np.full(2, lin(J)) for J in Js]), Js)
    s_full = integral_cross_section(E, mu, np.stack([np.full(2, lin(J)) for J in range(21)]))
    assert np.allclose(s_sparse, s_full, rtol=1e-14)
    with pytest.raises(ValueError):
        integral_cross_section(E, mu, P[:3], [0, 5, 3])
