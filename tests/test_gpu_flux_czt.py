"""The chirp-z form of the flux-to-energy accumulation (k_flux_czt): on an
energy grid E_0 + j dE, full chunks of the flux history are accumulated by FFT
convolutions instead of the direct sum over steps; both forms must give the
same P(E).  Energies off a uniform grid keep the direct form."""
import numpy as np
import pytest

from qd_b200 import Propagator
from qd_b200 import systems as S


def _case(prec, steps):
    d = S.case_c0(total_steps=steps)
    d.options.precision = prec
    return d


def _crp(d, steps, monkeypatch, czt):
    if czt:
        monkeypatch.delenv("QD_FLUX_CZT", raising=False)
    else:
        monkeypatch.setenv("QD_FLUX_CZT", "0")
    with Propagator(S.copy_case(d)) as p:
        p.propagate(steps)
        return p.crp()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_chirp_z_matches_direct_sum(prec, monkeypatch):
    # 620 steps: two full chunks of 250 in the chirp-z form, the last 120 direct
    d = _case(prec, 620)
    E = d.CRP.energies
    assert np.abs(np.diff(E) - (E[-1] - E[0]) / (E.size - 1)).max() < 1e-15
    a = _crp(d, 620, monkeypatch, czt=True)
    b = _crp(d, 620, monkeypatch, czt=False)
    scale = np.abs(b).max()
    assert scale > 0
    assert np.abs(a - b).max() < 1e-11 * scale + 1e-14


@pytest.mark.gpu
def test_nonuniform_energies_keep_the_direct_sum(monkeypatch):
    d = _case(0, 260)
    E = d.CRP.energies.copy()
    E[E.size // 2] += 1e-6 * (E[1] - E[0])      # off the grid: no chirp-z form
    d.CRP.energies = np.ascontiguousarray(E)
    a = _crp(d, 260, monkeypatch, czt=True)
    b = _crp(d, 260, monkeypatch, czt=False)
    assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_pe_fused_into_the_closing_accumulation(prec, monkeypatch):
    # a call that ends with a partial chunk: its GEMM-form accumulation also
    # sums P(E) per tile; the separate P(E) pass over phi_E must agree
    d = _case(prec, 140)
    out = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("QD_CRP_FUSED", fused)
        with Propagator(S.copy_case(d)) as p:
            p.propagate(70)
            first = p.crp()
            p.propagate(70)
            out[fused] = (first, p.crp())
    for a, b in zip(out["1"], out["0"]):
        scale = np.abs(b).max()
        assert scale > 0
        assert np.abs(a - b).max() < 1e-12 * scale + 1e-15
