"""The structured per-interval log (qd_b200.runlog) on a stand-in propagator:
record count and steps, norms, absorbed norm, energies, JSON lines."""
import io
import json
from types import SimpleNamespace

import numpy as np
import pytest

from qd_b200.runlog import propagate_logged


class FakePropagator:
    """Two runs whose norms fall by a fixed factor per step."""

    def __init__(self, steps=0):
        self.n_runs = 2
        self.data = SimpleNamespace(r1=SimpleNamespace(n=8), r2=SimpleNamespace(n=6),
                                    theta=SimpleNamespace(n=4))
        self.steps = steps
        self.hist = [[1.0 * 0.99 ** s, 2.0 * 0.98 ** s] for s in range(1, steps + 1)]
        self.every = 0
        self.log = []
        self.on_demand = 0

    def propagate(self, k):
        for _ in range(k):
            self.steps += 1
            s = self.steps
            self.hist.append([1.0 * 0.99 ** s, 2.0 * 0.98 ** s])
            if self.every and s % self.every == 0:
                self.log.append([s] + list(np.array([0.1, 0.2, 0.3, 0.6]) * s))

    def set_energy_interval(self, every):
        self.every = every

    def energy_log(self, run=0, cap=1 << 20):
        return np.array(self.log[-cap:]) if self.log else np.zeros((0, 5))

    def norms(self, n, run=0):
        if n > len(self.hist):
            raise RuntimeError("not available")
        return np.array([h[run] for h in self.hist[len(self.hist) - n:]])

    def energies(self, run=0):
        self.on_demand += 1
        return np.array([0.1, 0.2, 0.3, 0.6]) * self.steps


def test_records_per_interval():
    p = FakePropagator()
    out = io.StringIO()
    recs = propagate_logged(p, 25, 10, out, clock=iter(range(100)).__next__)
    assert [r["step"] for r in recs] == [10, 20, 25]
    assert [r["steps"] for r in recs] == [10, 10, 5]
    lines = [json.loads(x) for x in out.getvalue().splitlines()]
    assert lines == recs
    assert np.allclose(recs[-1]["norm"], [0.99 ** 25, 2.0 * 0.98 ** 25])
    # the second record's loss is counted from the first record's last norm
    assert np.allclose(recs[1]["absorbed"], [0.99 ** 10 - 0.99 ** 20,
                                              2.0 * (0.98 ** 10 - 0.98 ** 20)])
    # first record of a fresh handle: from the end of its first step
    assert np.allclose(recs[0]["absorbed"][0], 0.99 - 0.99 ** 10)
    assert recs[2]["energies"]["total"] == 0.6 * 25
    assert recs[0]["energies"]["kinetic"] == 0.1 * 10
    # steps 10 and 20 come from the in-propagation energies, step 25 on demand
    assert p.on_demand == 1 and [int(r[0]) for r in p.log] == [10, 20]
    assert p.every == 0                      # switched off again
    assert recs[0]["grid_pt_steps_per_s"] == 8 * 6 * 4 * 2 * 10 / 1


def test_unaligned_start_shortens_the_first_chunk():
    p = FakePropagator(steps=3)
    recs = propagate_logged(p, 20, 10, io.StringIO(), clock=iter(range(100)).__next__)
    assert [r["step"] for r in recs] == [10, 20, 23]
    assert [r["steps"] for r in recs] == [7, 10, 3]
    assert p.on_demand == 1


def test_resumed_handle_counts_from_its_last_step():
    p = FakePropagator(steps=5)
    recs = propagate_logged(p, 5, 5, io.StringIO(), energies=False,
                            clock=iter(range(10)).__next__)
    assert "energies" not in recs[0]
    assert np.allclose(recs[0]["absorbed"][1], 2.0 * (0.98 ** 5 - 0.98 ** 10))


@pytest.mark.gpu
def test_logged_propagation_on_gpu():
    from qd_b200 import systems as S, Propagator
    from oracle import pyoracle as O
    d = S.build_case("f+h2", 32, 24, 12, m=11, total_steps=30, n_energies=5,
                     n_gradient_points=5)
    a = S.copy_case(d)
    _, eref = O.oracle_time_evolution(a, energies=True)   # per step, as the reference prints
    out = io.StringIO()
    with Propagator(d) as p:
        recs = propagate_logged(p, 30, 10, out)
        allnorms = p.norms(30)
    assert [r["step"] for r in recs] == [10, 20, 30]
    assert recs[-1]["norm"][0] == allnorms[-1]
    assert recs[1]["absorbed"][0] == allnorms[9] - allnorms[19]
    for r in recs:
        e, ref = r["energies"], eref[r["step"] - 1]
        got = [e["kinetic"], e["rotational"], e["potential"], e["total"]]
        assert np.abs(np.array(got) - ref).max() <= 1e-10 * np.abs(ref).max()
    assert all(r["grid_pt_steps_per_s"] > 0 for r in recs)
