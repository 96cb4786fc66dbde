"""The BKMP2 H3 surface on the GPU (qd_bkmp2_*) against the oracle
restatement of H3/bkmp2.F (oracle/bkmp2_oracle.py)."""
import math

import numpy as np
import pytest

from oracle.bkmp2_oracle import VH2MIN, bkmp2
from qd_b200 import systems as S
from qd_b200.timeevolution import bkmp2_gpu, potential_bkmp2_gpu

pytestmark = pytest.mark.gpu


def _triangles(n, seed, lo=0.5, hi=6.0):
    rng = np.random.default_rng(seed)
    a = rng.uniform(lo, hi, n)
    b = rng.uniform(lo, hi, n)
    c = rng.uniform(np.maximum(np.abs(a - b) + 1e-3, lo), a + b - 1e-3)
    return a, b, c


def test_points_match_oracle():
    # including compact geometries (a distance below 1.15 bohr: the Cbend,
    # csym and casym terms) and near-collinear ones
    a, b, c = _triangles(600, 11, lo=0.45)
    got = bkmp2_gpu(a, b, c)
    ref = np.array([bkmp2(x, y, z) for x, y, z in zip(a, b, c)])
    assert np.all(np.isfinite(got))
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    assert (np.minimum(np.minimum(a, b), c) < 1.15).sum() > 100


def test_symmetric_and_invalid_on_gpu():
    a, b, c = _triangles(100, 5)
    v = bkmp2_gpu(a, b, c)
    for p in ((b, c, a), (c, a, b), (b, a, c)):
        assert np.abs(bkmp2_gpu(*p) - v).max() < 1e-13 * max(1.0, np.abs(v).max())
    bad = bkmp2_gpu([1.0, 0.15], [1.0, 2.0], [2.5, 2.0])
    assert np.all(np.isnan(bad))


def test_jacobi_grid_matches_oracle():
    masses = np.array([1.00783, 1.00783, 1.00783]) * S.AMU_ME
    R = np.linspace(0.5, 8.0, 18)
    r = np.linspace(0.4, 6.0, 12)
    x, _ = S.gauss_legendre(8)
    pot = potential_bkmp2_gpu(R, r, x, masses, vmax=2.5, rmin=0.4, cap=True)
    f2 = masses[2] / (masses[1] + masses[2])
    f3 = 1.0 - f2
    ref = np.empty_like(pot)
    for k, cth in enumerate(x):
        for j, rv in enumerate(r):
            for i, Rv in enumerate(R):
                r12 = math.sqrt((f2 * rv) ** 2 + Rv * Rv - 2.0 * f2 * rv * Rv * cth)
                r13 = math.sqrt((f3 * rv) ** 2 + Rv * Rv + 2.0 * f3 * rv * Rv * cth)
                v = 2.5
                if r12 > 0.4 and r13 > 0.4 and rv > 0.4:
                    v = min(bkmp2(r12, rv, r13) - VH2MIN, 2.5)
                ref[k, j, i] = v
    assert np.abs(pot - ref).max() < 1e-12
