"""Parity at the sizes of the benchmarked configurations.

* The plain FP64 form against the reference's own CPU propagator
  (common/timeEvol.C built in oracle/_ref against the shims; the C oracle,
  bit-exact to it, where that build is absent) on the full grids of the
  configurations: F + H2 J = 0 on 128 x 128 x 64 (C1), on 128 x 96 x 64 (the
  C2 grid, radix-3 in r) and on 256 x 192 x 128 (the C4 grid), 12 steps each;
  a centrifugal-sudden block (K > 0) of the C2 and of the C4 grid against the
  C oracle, whose rotational-phase index j = K + l is the one extension the
  reference lacks.  Tolerances: psi 1e-10 relative, norms 1e-10 relative,
  P(E) 1e-8 absolute.
* The complex64 form against the FP64 form on the whole batches that the
  benchmark times: the 64 centrifugal-sudden runs of C2 and the 32 blocks of
  C4, a few hundred steps: max |dP(E)| <= 1e-3 over energies where
  eta^2 > 1e-3 max eta^2 (the budget), psi 1e-3 relative, norms 1e-3 (the
  complex64 form loses about 1.4e-7 of the norm per step on the C4 grid with
  the tensor-core column pass, 1e-8 on the C2 grid, measured before any
  absorption; the P(E) budget holds).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from qd_b200 import systems as S, QD_PREC_FP32, QD_PREC_FP64
from qd_b200.timeevolution import Propagator

pytestmark = pytest.mark.gpu

PSI_REL = 1e-10
CRP_ABS = 1e-8
BUDGET = 1e-3


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _gpu(data, steps):
    b = S.copy_case(data)
    b.options.precision = QD_PREC_FP64
    with Propagator(b) as p:
        p.propagate(steps)
        norms = p.norms(steps)
        p.download()
    return b, norms


def _reference(data, steps):
    """The reference's own build when present (norms from the C oracle, which
    is bit-exact to it), else the C oracle."""
    a = S.copy_case(data)
    a.options.precision = QD_PREC_FP64
    a.time.total_steps = steps
    c = S.copy_case(a)
    norms, _ = O.oracle_time_evolution(c, norms=True)
    if O.ref_available() and int(getattr(getattr(data, "cs", None), "K", 0)) == 0:
        O.ref_time_evolution(a)
        return a, norms
    return c, norms


GRIDS = {
    "c1_128x128x64": dict(n1=128, n2=128, n_theta=64, m=63),
    "c2_128x96x64": dict(n1=128, n2=96, n_theta=64, m=63, r=(0.4, 8.0)),
    "c4_256x192x128": dict(n1=256, n2=192, n_theta=128, m=127, r=(0.4, 8.0)),
}
STEPS = 12


def _base(grid, steps):
    return S.build_case("f+h2", total_steps=steps, **GRIDS[grid])


@pytest.mark.parametrize("grid", list(GRIDS))
def test_fp64_full_grid_matches_reference(grid):
    base = _base(grid, STEPS)
    ref, norms = _reference(base, STEPS)
    got, gnorms = _gpu(base, STEPS)
    assert got.time.steps == ref.time.steps == STEPS
    assert rel(got.psi, ref.psi) < PSI_REL
    assert np.abs(gnorms - norms).max() < PSI_REL * norms.max()
    assert np.abs(got.CRP.CRP - ref.CRP.CRP).max() < CRP_ABS


@pytest.mark.parametrize("grid,J,K", [("c2_128x96x64", 10, 2), ("c4_256x192x128", 8, 3)])
def test_fp64_full_grid_cs_block_matches_oracle(grid, J, K):
    base = _base(grid, STEPS)
    run = S.cs_case(base, J, K, 0, 3)
    ref, norms = _reference(run, STEPS)
    got, gnorms = _gpu(run, STEPS)
    assert rel(got.psi, ref.psi) < PSI_REL
    assert np.abs(gnorms - norms).max() < PSI_REL * norms.max()
    assert np.abs(got.CRP.CRP - ref.CRP.CRP).max() < CRP_ABS


def _batch_pair(runs, steps):
    """(P(E), psi of run 0, norms) of the batch in complex64 and in FP64."""
    out = {}
    for prec in (QD_PREC_FP32, QD_PREC_FP64):
        rs = [S.copy_case(r) for r in runs]
        for r in rs:
            r.options.precision = prec
        with Propagator(rs) as p:
            p.propagate(steps)
            crp = np.stack([p.crp(i) for i in range(len(rs))])
            norms = np.stack([p.norms(steps, i) for i in range(len(rs))])
            psi0 = p.psi(0)
            psi_last = p.psi(len(rs) - 1)
        out[prec] = (crp, psi0, psi_last, norms)
    return out


def _check_budget(runs, out):
    c32, p32, q32, n32 = out[QD_PREC_FP32]
    c64, p64, q64, n64 = out[QD_PREC_FP64]
    worst = 0.0
    for i, r in enumerate(runs):
        eta = r.CRP.eta_sq
        sel = eta > 1e-3 * eta.max()
        worst = max(worst, float(np.abs(c32[i] - c64[i])[sel].max()))
    assert worst <= BUDGET, worst
    assert rel(p32, p64) < 1e-3
    assert rel(q32, q64) < 1e-3
    assert np.abs(n32 - n64).max() < 1e-3 * n64.max()
    return worst


def test_fp32_whole_c2_batch_within_budget():
    runs = S.case_c2(64, total_steps=600)
    assert len(runs) == 64
    _check_budget(runs, _batch_pair(runs, 600))


def test_fp32_whole_c4_batch_within_budget():
    runs = S.case_c4(32, total_steps=300)
    assert len(runs) == 32
    _check_budget(runs, _batch_pair(runs, 300))
