"""Run-level sharding of a batch over ranks, one process per GPU.

The propagations of a batch are independent: nothing is exchanged while they
step.  Rank r of W propagates runs r, r+W, r+2W, ... (round robin, so an
uneven tail spreads over the ranks) as one local batch on its own GPU, and the
per-run results -- time.steps and P(E), and psi if asked for -- are gathered to
every rank at the end with one all-gather of the host group
(qd_b200.hostgroup).  A single propagation is not split across GPUs (its
column and l-space passes would need two all-to-all transposes per step).
"""
from .hostgroup import FileGroup
from .timeevolution import TimeEvolutionMexCUDA


def shard(n_runs, rank, world):
    """Indices of the runs that `rank` of `world` propagates."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return list(range(rank, n_runs, world))


def time_evolution_sharded(runs, group=None, gather_psi=False, propagate=None):
    """Propagate `runs` (a list of structs, as for TimeEvolutionMexCUDA) over
    the ranks of `group` (a FileGroup; default: the job's group from the
    environment).  On return every rank holds time.steps and CRP.CRP of all
    runs, and psi of all runs if `gather_psi` (else only of its own).
    `propagate` runs one local batch in place (default: TimeEvolutionMexCUDA
    on this rank's GPU)."""
    group = group or FileGroup.from_env()
    propagate = propagate or TimeEvolutionMexCUDA
    mine = shard(len(runs), group.rank, group.world)
    local = [runs[i] for i in mine]
    if local:
        propagate(local)
    payload = [(i, int(runs[i].time.steps), runs[i].CRP.CRP.copy(),
                runs[i].psi.copy() if gather_psi else None) for i in mine]
    for part in group.allgather(payload):
        for i, steps, crp, psi in part:
            runs[i].time.steps = steps
            runs[i].CRP.CRP[:] = crp
            if psi is not None:
                runs[i].psi[...] = psi
    return runs
