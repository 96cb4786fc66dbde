"""The HSW surface of F + H2 on the GPU (qd_hsw_*) against the oracle
restatement of FH2/HSW/hswpot.F + sospline.F and the known answers of
FH2/HSW/verify.F."""
import math
import os

import numpy as np
import pytest

from oracle.hsw_oracle import SHIFT, HswOracle
from qd_b200 import systems as S
from qd_b200.timeevolution import HswSurface

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = dict(np.load(os.path.join(HERE, "golden", "hsw_tables.npz")))
KAT = [((2.0, 2.0, 2.0), 3.412633992079376e-02),
       ((4.0, 1.5, 4.5), 1.839160872060410e-03)]
MASSES = np.array([18.9984, 1.00783, 1.00783]) * S.AMU_ME


@pytest.fixture(scope="module")
def oracle():
    return HswOracle(TABLES)


def _points(n, seed):
    # Jacobi (R, r, gamma) of F + H2 covering the valley, the spline box edges
    # and the strong-interaction region
    rng = np.random.default_rng(seed)
    R = rng.uniform(1.0, 9.0, n)
    r = rng.uniform(0.9, 4.0, n)
    g = rng.uniform(0.0, math.pi, n)
    rhf1 = np.sqrt(R * R + 0.25 * r * r - R * r * np.cos(g))
    rhf2 = np.sqrt(R * R + 0.25 * r * r + R * r * np.cos(g))
    return rhf1, r, rhf2


def test_known_answers_on_gpu():
    with HswSurface(tables=TABLES) as h:
        for (x, y, z), v in KAT:
            got = float(h(x, y, z))
            # verify.F's values take the final 0.0006 in double precision; the
            # reference as built adds its single-precision value
            # (FP64 on the GPU: fused multiply-adds and the device exp differ from
            # the host's in the last bits)
            assert abs((got - (SHIFT - 0.0006)) - v) <= 1e-12 * abs(v), (got, v)


def test_points_match_oracle(oracle):
    a, b, c = _points(400, 7)
    with HswSurface(tables=TABLES) as h:
        got = h(a, b, c)
    ref = oracle.many(a, b, c)
    assert np.abs(got - ref).max() < 1e-13 * max(1.0, np.abs(ref).max())
    # the spin-orbit branch was taken for a good share of the points
    inside = 0
    for x, y, z in zip(a, b, c):
        v = oracle.sw1(x, y, z)
        rbig = math.sqrt(0.5 * (x * x + z * z - 0.5 * y * y))
        inside += v > oracle.esocut and y < oracle.rsolim and rbig > oracle.rrsolm
    assert inside > 50


def test_jacobi_grid_matches_oracle(oracle):
    R = np.linspace(0.8, 9.0, 20)
    r = np.linspace(0.6, 5.0, 14)
    x, _ = S.gauss_legendre(8)
    with HswSurface(tables=TABLES) as h:
        pot = h.potential(R, r, x, MASSES, vmax=2.5, rmin=0.4, cap=True)
    f2 = MASSES[2] / (MASSES[1] + MASSES[2])
    f3 = 1.0 - f2
    ref = np.empty_like(pot)
    for k, c in enumerate(x):
        for j, rv in enumerate(r):
            for i, Rv in enumerate(R):
                r12 = math.sqrt((f2 * rv) ** 2 + Rv * Rv - 2.0 * f2 * rv * Rv * c)
                r13 = math.sqrt((f3 * rv) ** 2 + Rv * Rv + 2.0 * f3 * rv * Rv * c)
                v = 2.5
                if r12 > 0.4 and r13 > 0.4 and rv > 0.4:
                    v = min(oracle.pot(r12, rv, r13), 2.5)
                ref[k, j, i] = v
    assert np.abs(pot - ref).max() < 1e-12


def test_data_directory_and_tables_agree(tmp_path):
    # the reference's four files written back from the fixture, read by qd_hsw_create
    t = TABLES
    with open(tmp_path / "three.param", "w") as f:
        for n, (i, j, k, a) in enumerate(zip(t["ix"], t["iy"], t["iz"], t["a"])):
            f.write(f"{n + 1:9d} {int(i):6d} {int(j):5d} {int(k):5d} {float(a):24.17e}\n")
    with open(tmp_path / "two.param", "w") as f:
        f.writelines(f"{float(v):.17g}\n" for v in t["p"])
    with open(tmp_path / "so.param", "w") as f:
        f.writelines(f" {float(v):.17g}      (comment)\n" for v in t["so_param"])
    nx, ny, nz = t["so"].shape
    with open(tmp_path / "so.input", "w") as f:
        f.write(f" {nx} {ny} {nz}\n")
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    f.write(" ".join(f"{float(v):.17g}" for v in
                                     (t["x"][i], t["y"][j], t["z"][k], t["so"][i, j, k])) + "\n")
    a, b, c = _points(200, 3)
    with HswSurface(str(tmp_path)) as h1, HswSurface(tables=t) as h2:
        assert np.array_equal(h1(a, b, c), h2(a, b, c))


def test_missing_directory_is_an_error(tmp_path):
    from qd_b200._abi import QdError
    with pytest.raises(QdError):
        HswSurface(str(tmp_path / "nowhere"))
