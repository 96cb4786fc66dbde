"""Run-level sharding over ranks (qd_b200.replicas) on CPU: two ranks as
separate processes meeting through the host file group, each propagating its
share of a batch with the CPU oracle standing in for its GPU, against the
same batch propagated serially; and a rank that never arrives."""
import multiprocessing as mp
import os
import tempfile

import numpy as np
import pytest

from qd_b200 import systems as S
from qd_b200.hostgroup import FileGroup
from qd_b200.replicas import shard

WORLD = 2


def _batch():
    base = S.build_case("h+h2", 16, 12, 8, m=7, total_steps=6, n_energies=5,
                        n_gradient_points=3)
    return S.batch_cases(base, [(0, 0), (0, 1), (1, 0), (0, 2), (1, 1)])


def _oracle_batch(runs):
    from oracle import pyoracle as O
    for r in runs:
        O.oracle_time_evolution(r)


def _rank_main(rank, group_dir, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "quantum-dynamics_b200")):
        sys.path.insert(0, p)
    from qd_b200.hostgroup import FileGroup
    from qd_b200.replicas import time_evolution_sharded
    group = FileGroup(rank, WORLD, group_dir, timeout=120)
    runs = _batch()
    time_evolution_sharded(runs, group=group, gather_psi=True, propagate=_oracle_batch)
    t = group.max(float(rank) + 0.5)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"),
             crp=np.stack([r.CRP.CRP for r in runs]),
             psi=np.stack([r.psi for r in runs]),
             steps=np.array([r.time.steps for r in runs]), tmax=t)


def test_shard_covers_every_run_once():
    for n in (1, 5, 64):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shard(n, r, w))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_two_ranks_match_serial_batch():
    ref = _batch()
    _oracle_batch(ref)
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as d:
        gd = os.path.join(d, "group")
        procs = [ctx.Process(target=_rank_main, args=(r, gd, d)) for r in range(WORLD)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        for rank in range(WORLD):
            z = np.load(os.path.join(d, f"rank{rank}.npz"))
            assert np.array_equal(z["steps"], [r.time.steps for r in ref])
            assert np.array_equal(z["crp"], np.stack([r.CRP.CRP for r in ref]))
            assert np.array_equal(z["psi"], np.stack([r.psi for r in ref]))
            assert float(z["tmax"]) == WORLD - 0.5


def test_missing_rank_ends_the_wait():
    with tempfile.TemporaryDirectory() as d:
        g = FileGroup(0, 2, d, timeout=0.3)
        with pytest.raises(TimeoutError):
            g.barrier()
