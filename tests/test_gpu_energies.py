"""Energies inside the propagation (qd_set_energy_interval): the step's own
kernels sum E_kin, E_rot and E_pot in FP64 on steps that are multiples of the
interval, at the points of the step where the reference prints them
(evolution_dt, common/timeEvol.C:619-647: kinetic after the kinetic phase,
rotational after the second Rot(dt/2), potential after the backward Legendre
transform, all before the absorber).  Checked against the CPU oracle's
per-step energies: FP64 form 1e-10 relative, complex64 form 1e-4, on each
column-pass and l-space kernel and on batches."""
import numpy as np
import pytest

from oracle import pyoracle as O
from qd_b200 import systems as S, QD_PREC_FP32, QD_PREC_FP64
from qd_b200.timeevolution import Propagator

pytestmark = pytest.mark.gpu

TOL = {QD_PREC_FP64: 1e-10, QD_PREC_FP32: 1e-4}


def _oracle_energies(data, steps):
    a = S.copy_case(data)
    a.options.precision = QD_PREC_FP64
    a.time.total_steps = steps
    _, e = O.oracle_time_evolution(a, energies=True)
    return e


def _check(log, eref, tol, steps_expected):
    assert [int(x) for x in log[:, 0]] == steps_expected
    for rec in log:
        ref = eref[int(rec[0]) - 1]
        assert np.abs(rec[1:] - ref).max() <= tol * np.abs(ref).max(), (rec, ref)


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
@pytest.mark.parametrize("shape", [(64, 64, 32), (128, 96, 64)])
def test_energy_interval_matches_oracle(prec, shape):
    n1, n2, nth = shape
    base = S.build_case("f+h2", n1, n2, nth, m=nth - 1, total_steps=24, n_energies=9,
                        precision=prec)
    eref = _oracle_energies(base, 24)
    d = S.copy_case(base)
    with Propagator(d) as p:
        p.set_energy_interval(4)
        p.propagate(10)            # 4, 8 in this call
        p.propagate(14)            # 12 .. 24: the call boundary falls between energy steps
        log = p.energy_log()
    _check(log, eref, TOL[prec], [4, 8, 12, 16, 20, 24])


@pytest.mark.parametrize("env", [{"QD_SLICE_CLUSTER": "0"}, {"QD_SLICE_CLUSTER": "1"},
                                 {"QD_SLICE_CLUSTER": "9"}, {"QD_COLUMN_PATH": "simt"}],
                         ids=lambda e: "-".join(f"{k}={v}" for k, v in e.items()))
def test_energy_interval_on_each_kernel(env, monkeypatch):
    # split l-space kernels, the Stockham cluster kernel (whose energy steps
    # run on the split kernels), the 2-CTA register-FFT kernel, the SIMT
    # column pass (plain l-space basis)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    base = S.build_case("f+h2", 128, 96, 64, m=63, total_steps=12, n_energies=9,
                        precision=QD_PREC_FP32)
    eref = _oracle_energies(base, 12)
    d = S.copy_case(base)
    with Propagator(d) as p:
        p.set_energy_interval(3)
        p.propagate(12)
        log = p.energy_log()
    _check(log, eref, 1e-4, [3, 6, 9, 12])


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_energy_interval_on_a_cs_batch(prec):
    base = S.build_case("f+h2", 64, 64, 32, m=31, total_steps=10, n_energies=9)
    runs = [S.cs_case(base, J, K, 0, 2) for J, K in ((0, 0), (4, 1), (6, 2))]
    for r in runs:
        r.options.precision = prec
    refs = [_oracle_energies(r, 10) for r in runs]
    with Propagator([S.copy_case(r) for r in runs]) as p:
        p.set_energy_interval(5)
        p.propagate(10)
        for i in range(len(runs)):
            _check(p.energy_log(i), refs[i], TOL[prec], [5, 10])


def test_energy_interval_off_records_nothing():
    base = S.build_case("h+h2", 32, 32, 16, m=15, total_steps=6, n_energies=5)
    with Propagator(S.copy_case(base)) as p:
        p.propagate(6)
        assert len(p.energy_log()) == 0
        p.set_energy_interval(2)
        p.propagate(4)              # steps 7 .. 10: energies at 8 and 10
        assert [int(x) for x in p.energy_log()[:, 0]] == [8, 10]
