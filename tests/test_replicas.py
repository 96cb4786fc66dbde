"""Run-level sharding over ranks (qd_b200.replicas) on CPU: two gloo ranks,
each propagating its share of a batch with the CPU oracle standing in for its
GPU, against the same batch propagated serially."""
import os
import socket
import tempfile

import numpy as np
import pytest

from qd_b200 import systems as S
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


def _rank_main(rank, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "quantum-dynamics_b200")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from qd_b200.replicas import time_evolution_sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=WORLD)
    try:
        runs = _batch()
        time_evolution_sharded(runs, gather_psi=True, propagate=_oracle_batch)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"),
                 crp=np.stack([r.CRP.CRP for r in runs]),
                 psi=np.stack([r.psi for r in runs]),
                 steps=np.array([r.time.steps for r in runs]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_run_once():
    for n in (1, 5, 64):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shard(n, r, w))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_two_gloo_ranks_match_serial_batch():
    import torch.multiprocessing as mp
    ref = _batch()
    _oracle_batch(ref)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(_free_port(), d), nprocs=WORLD, join=True,
                           start_method="spawn")
        for rank in range(WORLD):
            z = np.load(os.path.join(d, f"rank{rank}.npz"))
            assert np.array_equal(z["steps"], [r.time.steps for r in ref])
            assert np.array_equal(z["crp"], np.stack([r.CRP.CRP for r in ref]))
            assert np.array_equal(z["psi"], np.stack([r.psi for r in ref]))
