"""The periodic copy-back of the drop-in entry point: with
options.steps_to_copy_psi_from_device_to_host = N, qd_time_evolution writes
psi, time.steps and P(E) into the caller's struct every N steps and calls the
progress callback (the reference's GPU loop, common-cuda/evolutionCUDA2.cu:
540-546).  Checked through the C ABI against the CPU oracle run for the same
number of steps."""
import numpy as np
import pytest

from qd_b200 import systems as S, TimeEvolutionMexCUDA, QD_PREC_FP32, QD_PREC_FP64
from qd_b200._abi import PROGRESS_FN, QD_ERR_STOPPED, QdError

pytestmark = pytest.mark.gpu

TOL = {QD_PREC_FP64: (1e-10, 1e-8), QD_PREC_FP32: (1e-4, 1e-6)}


def _case(prec, steps):
    return S.build_case("f+h2", 32, 32, 16, m=15, total_steps=steps, n_energies=9,
                        precision=prec)


def _oracle(base, steps):
    from oracle import pyoracle as O
    a = S.copy_case(base)
    a.options.precision = QD_PREC_FP64
    a.time.total_steps = steps
    norms, _ = O.oracle_time_evolution(a, norms=True)
    return a, norms


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_progress_every_n_steps_matches_oracle(prec):
    base = _case(prec, 30)
    d = S.copy_case(base)
    d.options.steps_to_copy_psi_from_device_to_host = 10
    seen = []

    def cb(step, norm, psi, ctx):
        seen.append((step, norm, C_addr(psi) == d.psi.ctypes.data, d.psi.copy(),
                     d.CRP.CRP.copy()))
        return 0

    d.options.progress = PROGRESS_FN(cb)
    TimeEvolutionMexCUDA(d)
    assert [s[0] for s in seen] == [10, 20, 30]
    assert d.time.steps == 30
    psi_tol, crp_tol = TOL[prec]
    _, norms = _oracle(base, 30)
    for step, norm, same_array, psi, crp in seen:
        ref, _ = _oracle(base, step)
        assert same_array                      # the callback sees the caller's array
        assert _rel(psi, ref.psi) < psi_tol
        assert np.abs(crp - ref.CRP.CRP).max() < crp_tol
        assert abs(norm - norms[step - 1]) < psi_tol * norms[0]
    assert _rel(d.psi, seen[-1][3]) == 0.0


def C_addr(p):
    import ctypes
    return ctypes.cast(p, ctypes.c_void_p).value


def test_progress_can_stop_the_call():
    base = _case(QD_PREC_FP64, 40)
    d = S.copy_case(base)
    d.options.steps_to_copy_psi_from_device_to_host = 7
    steps = []

    def cb(step, norm, psi, ctx):
        steps.append(step)
        return 1 if step == 14 else 0

    d.options.progress = PROGRESS_FN(cb)
    with pytest.raises(QdError) as e:
        TimeEvolutionMexCUDA(d)
    assert e.value.code == QD_ERR_STOPPED
    assert steps == [7, 14]
    assert d.time.steps == 14
    ref, _ = _oracle(base, 14)
    assert _rel(d.psi, ref.psi) < 1e-10
    assert np.abs(d.CRP.CRP - ref.CRP.CRP).max() < 1e-8


def test_copy_back_without_callback_ends_on_the_last_step():
    # 25 steps with N = 10: copies at 10 and 20, then the final state at 25
    base = _case(QD_PREC_FP64, 25)
    d = S.copy_case(base)
    d.options.steps_to_copy_psi_from_device_to_host = 10
    TimeEvolutionMexCUDA(d)
    ref, _ = _oracle(base, 25)
    assert d.time.steps == 25
    assert _rel(d.psi, ref.psi) < 1e-10
    assert np.abs(d.CRP.CRP - ref.CRP.CRP).max() < 1e-8
