"""J-summed quantities from centrifugal-sudden blocks (the consumer of a
batch of (J, K) propagations).  No counterpart in the reference, which
propagates J = 0 only.

For an initial diatom state (v0, j0) the centrifugal-sudden reaction
probability of total angular momentum J is the average over the 2 j0 + 1
projections K of j0 (P depends on |K| only):
    P_J(E) = (P_{J,0} + 2 sum_{K=1}^{min(J, j0)} P_{J,K}) / (2 j0 + 1),
and the integral cross section
    sigma(E) = pi / k^2 sum_J (2J + 1) P_J(E),   k^2 = 2 mu_R E_coll,
with J summed over every integer up to J_max; when only some J are
propagated, P_J is interpolated linearly between them (J-shifting-free
linear interpolation, the usual practice for sparse J grids).
"""
import numpy as np


def k_averaged(blocks, J, j0):
    """P_J(E) from the blocks {K: P_{J,K}(E)} of one J (missing K > j0 are
    zero: the initial state has no such projection)."""
    kmax = min(J, j0)
    tot = np.asarray(blocks[0], dtype=np.float64).copy()
    for K in range(1, kmax + 1):
        tot += 2.0 * np.asarray(blocks[K], dtype=np.float64)
    return tot / (2 * j0 + 1)


def integral_cross_section(e_coll, mu_R, P_of_J, j_values=None):
    """sigma(E) in bohr^2 from P_J(E) given at the total angular momenta
    j_values (ascending; default 0, 1, 2, ...), summing (2J+1) P_J over every
    integer J from 0 to the last one, P_J linear between the given J."""
    P = np.asarray(P_of_J, dtype=np.float64)
    Js = np.arange(P.shape[0]) if j_values is None else np.asarray(j_values)
    if np.any(np.diff(Js) <= 0) or Js[0] != 0:
        raise ValueError("j_values must ascend from 0")
    total = np.zeros(P.shape[1])
    for J in range(int(Js[-1]) + 1):
        i = np.searchsorted(Js, J)
        if Js[i] == J:
            pj = P[i]
        else:
            a = (J - Js[i - 1]) / (Js[i] - Js[i - 1])
            pj = (1 - a) * P[i - 1] + a * P[i]
        total += (2 * J + 1) * pj
    k2 = 2.0 * mu_R * np.asarray(e_coll, dtype=np.float64)
    return np.pi / k2 * total
