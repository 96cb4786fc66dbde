"""qd_energies_noalloc -- energies with the DFT scratch and the sums in a
static device array (no device allocation) -- against the allocating entry
point qd_energies_run, both called through the C ABI.

Collected last on purpose, so that a run that stops at the first failure has
run every other test first.  In a full run these cases follow the other
tests in the same process; test_noalloc_first_call_in_a_fresh_process runs
the entry point in a new process, where its first call on the device looks
up the static scratch's address.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from qd_b200 import _abi, systems as S, QD_PREC_FP32, QD_PREC_FP64
from qd_b200.timeevolution import Propagator

pytestmark = pytest.mark.gpu

MAX_POINTS = 1048576          # QD_ENERGIES_NOALLOC_MAX_POINTS of include/qd.h
REL = 1e-12                   # FP64 sums; only the atomicAdd order differs


def energies(fn, p, run):
    out = np.zeros(4)
    _abi.check(fn(p._h, run, out.ctypes.data_as(_abi.c_double_p)))
    return out


def assert_close(a, b):
    assert np.abs(a - b).max() <= REL * np.abs(b).max(), (a, b)


@pytest.mark.parametrize("prec", [QD_PREC_FP64, QD_PREC_FP32])
def test_noalloc_matches_allocating_twice_in_a_row(prec):
    L = _abi.lib()
    base = S.build_case("f+h2", 48, 40, 24, m=17, total_steps=30, n_energies=5,
                        precision=prec)
    with Propagator(base) as p:
        p.propagate(15)
        ref = energies(L.qd_energies_run, p, 0)
        first = energies(L.qd_energies_noalloc, p, 0)
        second = energies(L.qd_energies_noalloc, p, 0)   # the sums start from zero again
        assert_close(first, ref)
        assert_close(second, ref)
        p.propagate(15)
        ref2 = energies(L.qd_energies_run, p, 0)
        assert_close(energies(L.qd_energies_noalloc, p, 0), ref2)
        assert_close(energies(L.qd_energies_noalloc, p, 0), ref2)
        assert np.abs(ref2 - ref).max() > 0          # the state moved between the pairs


def test_noalloc_batch_runs():
    L = _abi.lib()
    base = S.build_case("f+h2", 32, 32, 16, m=15, total_steps=10, n_energies=5,
                        precision=QD_PREC_FP64)
    runs = S.batch_cases(base, [(0, 0), (0, 2), (1, 0)])
    with Propagator(runs) as p:
        p.propagate(10)
        for r in range(len(runs)):
            ref = energies(L.qd_energies_run, p, r)
            assert_close(energies(L.qd_energies_noalloc, p, r), ref)
            assert_close(energies(L.qd_energies_noalloc, p, r), ref)


def test_noalloc_rejects_grids_above_the_static_scratch():
    L = _abi.lib()
    d = S.build_case("h+h2", 128, 128, 72, m=40, total_steps=1, n_energies=3,
                     precision=QD_PREC_FP64)
    assert 128 * 128 * 72 > MAX_POINTS
    with Propagator(d) as p:
        out = np.zeros(4)
        rc = L.qd_energies_noalloc(p._h, 0, out.ctypes.data_as(_abi.c_double_p))
        assert rc == _abi.QD_ERR_INVALID
        assert b"static scratch" in L.qd_last_error()
        assert np.all(out == 0)
        # the allocating entry point still serves this size
        e = energies(L.qd_energies_run, p, 0)
        assert np.all(np.isfinite(e))


FRESH = r"""
import sys
import numpy as np
sys.path[:0] = [{repo!r}, {pkg!r}]
from qd_b200 import _abi, systems as S, QD_PREC_FP64
from qd_b200.timeevolution import Propagator, set_device
set_device(0)
L = _abi.lib()
base = S.build_case("f+h2", 48, 40, 24, m=23, total_steps=12, n_energies=5,
                    precision=QD_PREC_FP64)
with Propagator(base) as p:
    p.propagate(12)
    out = []
    for fn in (L.qd_energies_noalloc, L.qd_energies_noalloc, L.qd_energies_run):
        e = np.zeros(4)
        _abi.check(fn(p._h, 0, e.ctypes.data_as(_abi.c_double_p)))
        out.append(e)
for e in out[:2]:
    assert np.abs(e - out[2]).max() <= 1e-12 * np.abs(out[2]).max(), (e, out[2])
print("fresh-process noalloc ok")
"""


def test_noalloc_first_call_in_a_fresh_process():
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    code = FRESH.format(repo=repo, pkg=os.path.join(repo, "quantum-dynamics_b200"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process noalloc ok" in r.stdout
