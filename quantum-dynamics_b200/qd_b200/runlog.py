"""Structured per-interval log of a propagation, one JSON object per line.

The reference prints, after every step, the step index, the energies, the
wavepacket norm and the step's wall and CPU times (common/timeEvol.C:654-683).
Here the propagation runs on the device in chunks of `interval` steps and one
record is written per chunk:

    {"step": 400, "steps": 100, "seconds": 0.0025, "grid_pt_steps_per_s": 4.2e10,
     "norm": [0.99, ...], "absorbed": [1.2e-4, ...],
     "energies": {"kinetic": ..., "rotational": ..., "potential": ..., "total": ...}}

`norm` is the FP64 norm of every run after the chunk's last step and
`absorbed` the norm each run lost during the chunk (through the absorbers
only: the propagator is unitary otherwise), counted from the norm after the
previous record's last step, or, for the first record of a handle that has
made no step before, from the end of the chunk's first step; `energies` are those of run 0
after the chunk's last step, in hartree, summed on the device in FP64 by the
step's own kernels (qd_set_energy_interval; chunks end on multiples of
`interval`, the first one shortened to reach one) or, for a last chunk that
ends elsewhere, by the on-demand energies path (omitted with energies=False).
The time is the wall clock around the chunk, which ends when the chunk's norms
are back on the host.
"""
import json
import time


def propagate_logged(prop, n_steps, interval, out, energies=True, clock=time.perf_counter):
    """Advance `prop` (a Propagator) by n_steps in chunks of `interval` steps,
    writing one JSON line per chunk to the text stream `out`.  Returns the
    list of records."""
    if interval < 1:
        raise ValueError("interval must be >= 1")
    runs = prop.n_runs
    d = prop.data
    points = int(d.r1.n) * int(d.r2.n) * int(d.theta.n) * runs
    records = []
    prev = None
    if prop.steps > 0:
        try:
            prev = [float(prop.norms(1, r)[0]) for r in range(runs)]
        except Exception:           # no norm recorded by this handle yet
            prev = None
    if energies:
        prop.set_energy_interval(interval)
    done = 0
    while done < n_steps:
        k = min(interval - prop.steps % interval, n_steps - done)
        t0 = clock()
        prop.propagate(k)
        norms = [prop.norms(k, r) for r in range(runs)]
        dt = clock() - t0
        done += k
        first = [float(n[0]) for n in norms]
        last = [float(n[-1]) for n in norms]
        start = prev if prev is not None else first
        rec = {"step": int(prop.steps), "steps": k, "seconds": dt,
               "grid_pt_steps_per_s": points * k / dt if dt > 0 else None,
               "norm": last, "absorbed": [a - b for a, b in zip(start, last)]}
        if energies:
            log = prop.energy_log(0, 1)
            if len(log) and int(log[-1][0]) == prop.steps:
                e = log[-1][1:]
            else:
                e = prop.energies(0)
            rec["energies"] = {"kinetic": float(e[0]), "rotational": float(e[1]),
                               "potential": float(e[2]), "total": float(e[3])}
        out.write(json.dumps(rec) + "\n")
        out.flush()
        records.append(rec)
        prev = last
    if energies:
        prop.set_energy_interval(0)
    return records
