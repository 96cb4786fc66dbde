"""Benchmark: grid-point * steps / s of the split-operator propagator.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1|c0|c2|c2j0|c3|c4]

Workload (default c1): F + H2, J = 0, extended-LEPS surface on a
128 x 128 x 64 Jacobi grid (n_l = 64), complex64 wavefunction with the
3xTF32 Legendre GEMM and FP64 flux-to-P(E) accumulation, dt = 10 au; P(E)
on 241 energies, 11-point flux stencil.  A step is one split-operator step
of the whole grid (1,048,576 grid points) including the flux capture.

value   device time (CUDA events on the library's stream) of K steps after
        W warm-up steps, L2 flushed before every step outside the timed spans
        (256 MiB written, then read back, so the step meets neither its own
        data nor dirty lines in L2); whole-job = sum over ranks' points / max
        rank time.
e2e     the drop-in entry point qd_time_evolution on host arrays for the
        same K steps: upload of pot and psi, table set-up, the K steps, P(E)
        and the download of psi and P(E), wall clock.
Multi-GPU: independent replicas (one propagation per rank, weak scaling,
no data-path collective); rank times are reduced with MAX.

--impl reference times the reference's own CPU propagator (common/timeEvol.C,
built in oracle/_ref against the shims) on the host cores for a bounded
sample of steps of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "quantum-dynamics_b200"))

import numpy as np  # noqa: E402

METRIC = "grid-pt*steps/s"
FLUSH_BYTES = 256 << 20


EXTRA = {}


def surrogate_c1(precision, n_train=200000, steps=60000, seed=12345):
    """C1 with the potential replaced by the MLP surrogate: training on the GPU,
    the judge's |dV| on the grid, and |dP(E)| of two full 10000-step complex64
    propagations (plain LEPS vs surrogate)."""
    from qd_b200 import systems as S
    from qd_b200.surrogate import Surrogate, training_set, judge
    from qd_b200.timeevolution import Propagator, potential_jacobi
    data = S.case_c1(precision=precision)
    m_amu = np.array([18.9984, 1.00783, 1.00783]) * S.AMU_ME
    pes = S.leps_f_h2()
    R, r, x = data.r1.r, data.r2.r, data.theta.x
    r12, r23, r13, V = training_set(pes, m_amu, n=n_train, seed=seed)
    sur = Surrogate(seed=seed)
    t0 = time.perf_counter()
    loss = sur.fit(r12, r23, r13, V, steps=steps, lr=2e-3, lr_end=1e-6)
    t_train = time.perf_counter() - t0
    sur.potential(R, r, x, m_amu)
    t0 = time.perf_counter()
    pot = sur.potential(R, r, x, m_amu)
    t_grid = time.perf_counter() - t0
    t0 = time.perf_counter()
    potential_jacobi(R, r, x, m_amu, pes)
    t_plain = time.perf_counter() - t0
    rms, mx, _, plain = judge(sur, pes, R, r, x, m_amu)
    crp = []
    for p_ in (plain, pot):
        d = S.copy_case(data)
        d.pot = np.ascontiguousarray(p_)
        d.options.precision = 1
        with Propagator(d) as pr:
            pr.propagate(10000)
            crp.append(pr.crp())
    eta = data.CRP.eta_sq
    sel = eta > 1e-3 * eta.max()
    sur.close()
    out = S.copy_case(data)
    out.pot = np.ascontiguousarray(pot)
    info = {"n_train": int(r12.size), "adam_steps": steps, "batch": 4096,
            "train_seconds": t_train, "final_loss_std_units": loss,
            "dV_rms_meV": rms * S.HARTREE_EV * 1e3, "dV_max_meV": mx * S.HARTREE_EV * 1e3,
            "dV_region": "grid points where the plain LEPS is below 3 eV",
            "max_abs_dP_10000_steps": float(np.abs(crp[0] - crp[1])[sel].max()),
            "grid_eval_seconds_gpu_mlp": t_grid,
            "grid_eval_seconds_plain_pes_host_callback": t_plain}
    return out, info


def as_runs(data):
    """A workload is one run (a data struct) or a batch (a list of them)."""
    return list(data) if isinstance(data, (list, tuple)) else [data]


def grid_points(data):
    """Grid points of all runs of a workload."""
    return sum(int(d.r1.n) * int(d.r2.n) * int(d.theta.n) for d in as_runs(data))


def copy_workload(data):
    from qd_b200 import systems as S
    runs = [S.copy_case(d) for d in as_runs(data)]
    return runs if isinstance(data, (list, tuple)) else runs[0]


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_workload(name, precision, runs=64):
    from qd_b200 import systems as S
    if name == "c1":
        data = S.case_c1(precision=precision)
        desc = ("F+H2 J=0 extended-LEPS, 128x128x64 Jacobi grid, n_l=64, dt=10 au, "
                "241 energies, 11-point flux")
    elif name == "c0":
        data = S.case_c0(precision=precision)
        desc = "H+H2 J=0 extended-LEPS, 64x64x40 Jacobi grid, n_l=39, dt=10 au, 241 energies"
    elif name == "c3":
        data, info = surrogate_c1(precision)
        EXTRA["surrogate"] = info
        desc = ("F+H2 J=0 on the MLP surrogate of the extended-LEPS surface (trained on the GPU "
                f"on {info['n_train']} LEPS-labelled geometries), 128x128x64 Jacobi grid, n_l=64, "
                "dt=10 au, 241 energies")
    elif name == "c2":
        data = S.case_c2(runs, precision=precision)
        desc = (f"batch of {runs} F+H2 centrifugal-sudden blocks (J in 0,5,10,15,20; "
                "K <= min(J,4); n_j = 64 - K) x initial (v0,j0) in (0,0),(0,1),(0,2),(1,0), "
                "128x96x64 Jacobi grid, dt=10 au, 241 energies each")
    elif name == "c4":
        data = S.case_c4(min(runs, 32), precision=precision)
        desc = (f"batch of {min(runs, 32)} F+H2 centrifugal-sudden blocks (J in 0,4,..,28 with "
                "K <= min(J,3), then J=30 with K <= 2; n_j = 128 - K) from (v0,j0) = (0,3), "
                "256x192x128 Jacobi grid, dt=10 au, 241 energies each; extended-LEPS surface "
                "(the surface does not enter the step's arithmetic)")
    elif name == "c2j0":
        data = S.case_c2_j0(runs, precision=precision)
        desc = (f"batch of {runs} F+H2 J=0 propagations, 128x96x64 Jacobi grid, n_l=64, dt=10 au, "
                "initial (v0,j0) cycling (0,0),(0,1),(0,2),(1,0), 241 energies each")
    else:
        raise SystemExit(f"unknown workload {name}")
    return data, desc


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_rate(data, max_seconds, steps_cap=None):
    """Time the reference CPU propagator (oracle/_ref) -- or, if it was not
    built, the C oracle port -- on this workload: 1 warm-up step, then as many
    steps as fit in about max_seconds.  Returns (rate, info)."""
    from oracle import pyoracle as O
    from qd_b200 import systems as S
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    use_ref = O.ref_available()
    run = O.ref_time_evolution if use_ref else O.oracle_time_evolution
    runs = as_runs(data)
    d = S.copy_case(runs[0])
    d.options.precision = 0
    d.time.total_steps = 1
    t0 = time.perf_counter()
    run(d)
    t_step = time.perf_counter() - t0
    n = max(1, int(max_seconds / max(t_step, 1e-6)))
    if steps_cap:
        n = min(n, steps_cap)
    d.time.total_steps = n
    t0 = time.perf_counter()
    run(d)
    dt = time.perf_counter() - t0
    pts = grid_points(runs[0])
    what = "the same workload" if len(runs) == 1 else f"run 0 of the {len(runs)}-run batch"
    info = {"kind": "reference" if use_ref else "port", "cores": threads,
            "sample": f"{n} steps (after 1 warm-up step) of {what} in FP64, "
                      f"per-step energies/norm/CRP diagnostics included as in the reference"}
    return pts * n / dt, info


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        return rank, world, local, dist
    return rank, world, local, None


def run_reference(args):
    rank, world, local, dist = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    data, desc = build_workload(args.workload, 0, args.runs)
    budget = float(os.environ.get("QD_REF_SECONDS", "60"))
    rate, info = cpu_reference_rate(data, budget)
    pts = grid_points(data)
    info["value"] = rate
    info["unit"] = METRIC
    line = {"metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": pts / rate * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "grid_points": pts, "precision": "FP64 (reference CPU)"},
            "cpu_baseline": info,
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_ours(args):
    rank, world, local, dist = dist_setup(args.gpus)
    from qd_b200 import QD_PREC_FP32, QD_PREC_FP64, Propagator, TimeEvolutionMexCUDA
    from qd_b200 import systems as S
    from qd_b200.timeevolution import kernel_launch_count, set_device
    set_device(local)
    prec = QD_PREC_FP64 if args.fp64 else QD_PREC_FP32
    data, desc = build_workload(args.workload, prec, args.runs)
    runs = as_runs(data)
    pts = grid_points(data)
    K, W = args.steps, args.warmup

    # --- device-resident throughput -------------------------------------------------
    d = copy_workload(data)
    with Propagator(d) as p:
        p.propagate_timed(W, FLUSH_BYTES)
        if dist:
            dist.barrier()
        l0 = kernel_launch_count()
        with ClockSampler(local) as clk:
            ms = p.propagate_timed(K, FLUSH_BYTES)
        launches = kernel_launch_count() - l0
        # per-kernel-class device time (separate, profiled run)
        from qd_b200 import _abi
        import ctypes as C
        lib = _abi.lib()
        lib.qd_set_profiling(p._h, 1)
        p.propagate(min(K, 400))
        buf = (C.c_double * 10)()
        nw = C.c_int32()
        lib.qd_kernel_times(p._h, buf, 10, C.byref(nw))
        lib.qd_set_profiling(p._h, 0)
        kclass = list(buf)[:nw.value]
        # unflushed (L2-resident steady state), for context
        ms_warm = p.propagate_timed(K, 0)
    t_max = ms
    if dist:
        import torch
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = pts * K * world / (t_max * 1e-3)

    # --- end to end through the drop-in entry point -------------------------------
    # five repetitions, median reported (each a full call: upload, set-up, K steps,
    # P(E), download)
    reps = []
    for _ in range(5):
        e = copy_workload(data)
        for r in as_runs(e):
            r.time.total_steps = K
            r.time.steps = 0
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        TimeEvolutionMexCUDA(e)
        reps.append(time.perf_counter() - t0)
    e2e_s = float(np.median(reps))
    if dist:
        import torch
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = sum(r.pot.nbytes + r.psi.nbytes for r in runs) + runs[0].theta.legendre.nbytes
    d2h = sum(r.psi.nbytes + r.CRP.CRP.nbytes for r in runs)
    e2e = {"value": pts * K * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
           "seconds": e2e_s, "seconds_each": reps,
           "entry_point": "qd_time_evolution (TimeEvolutionMexCUDA), median of 5 calls"}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # --- roofline of the dominant kernel class ----------------------------------------
    peak, peak_kind = load_peaks()
    r0 = runs[0]
    nl, nth = int(r0.theta.m) + 1, int(r0.theta.n)
    n12 = int(r0.r1.n) * int(r0.r2.n) * len(runs)
    cb = 16 if args.fp64 else 8        # bytes per complex
    shared_pot = all(np.array_equal(r.pot, r0.pot) for r in runs[1:])
    npot = 1 if shared_pot else len(runs)
    alg = {  # algorithmic bytes per launch: psi_l read + written, exp(-iV dt) read once
        "column": n12 * 2 * nl * cb + int(r0.r1.n) * int(r0.r2.n) * nth * cb * npot,
        "lines": n12 * nl * 2 * cb,
    }
    # DRAM bytes (read + write) per launch from one ncu capture each (cold caches:
    # ncu flushes them before every captured launch); the batch figures were
    # captured on 32 (c2j0) or 4 (c4) runs and scale with the runs.  Sources: the
    # ncu summaries column_tc_and_slice_rf2_c1_128x128x64.md,
    # column_tc_and_slice_rf_batch32_128x96x64.md and
    # column_tc_and_slice_rf4_c4_4runs_256x192x128.md under profiles/.
    traffic_ncu = {("c1", "column"): 16.89e6, ("c1", "lines"): 9.30e6,
                   ("c2j0", "column"): 373.7e6 / 32, ("c2j0", "lines"): 379.7e6 / 32,
                   ("c4", "column"): 568.4e6 / 4, ("c4", "lines"): 360.6e6 / 4}
    names = ["column", "lines", "flux_prep", "flux_accum", "crp"]
    per = {names[i]: kclass[i] for i in range(min(5, len(kclass)))}
    step_ms = t_max / K
    dom = max(("column", "lines"), key=lambda k: per.get(k, 0.0))
    dom_ms = per.get(dom, float("nan"))
    achieved = alg[dom] / (dom_ms * 1e-3) / 1e9 if dom_ms and dom_ms > 0 else None
    tr = traffic_ncu.get((args.workload, dom)) if not args.fp64 else None
    if tr is not None and args.workload in ("c2j0", "c4"):
        tr *= len(runs)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": tr, "traffic_unit": "bytes per launch (ncu)",
                "alg_bytes_per_launch": alg[dom], "avg_launch_ms": dom_ms,
                "kernel_class_ms": per}

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        rate, info = cpu_reference_rate(data, float(os.environ.get("QD_CPU_SECONDS", "20")))
        info["value"] = rate
        info["unit"] = METRIC
        cpu = info
    curves_per_hour = 3600.0 / (e2e_s / K * 10000) if args.workload == "c1" else None
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32", "data": "synthetic",
            "config": {"workload": desc, "grid_points": pts,
                       "precision": "FP64 plain" if args.fp64 else
                       "complex64 + 3xTF32 Legendre + FP64 flux accumulation",
                       "l2": "flushed before every step (256 MiB write, then read back so no dirty lines remain; outside the timed spans)",
                       "parallelism": f"replicas x{world}"},
            "value_l2_resident": pts * K / (ms_warm * 1e-3),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clk.summary(), "gpu_launches": launches, **EXTRA,
            "pe_curves_per_hour_e2e": curves_per_hour}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c0", "c2", "c2j0", "c3", "c4"])
    ap.add_argument("--runs", type=int, default=64, help="runs of the c2j0 batch")
    ap.add_argument("--fp64", action="store_true", help="plain FP64 form instead of complex64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
