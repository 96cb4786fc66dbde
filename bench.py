"""Benchmark: grid-point * steps / s of the split-operator propagator.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c4|c2|c2j0|c1|c0|c3]

Workload (default c4, the largest single-GPU configuration): a batch of 32
F + H2 centrifugal-sudden blocks (J = 0-30, K <= 3, n_j = 128 - K) on a
256 x 192 x 128 Jacobi grid, 201,326,592 grid points, complex64 wavefunction
with the 3xFP16 Legendre GEMM and FP64 flux-to-P(E) accumulation, dt = 10 au,
P(E) on 241 energies per block.  c2 is the 64-block batch on 128 x 96 x 64,
c1 one F + H2 J = 0 run on 128 x 128 x 64.  A step is one split-operator
step of every grid point of the workload, including the flux capture.

value   device time (CUDA events on the library's stream) of K steps after
        W warm-up steps, L2 flushed before every step outside the timed spans
        (256 MiB written, then read back, so the step meets neither its own
        data nor dirty lines in L2); whole-job = sum over ranks' points / max
        rank time.
fp64_plain  the plain FP64 form's rate on the same workload, timed the same
        way, and value / that rate.
e2e     the drop-in entry point qd_time_evolution on host arrays for the
        same K steps: upload of pot and psi, table set-up, the K steps, P(E)
        and the download of psi and P(E), wall clock.
clocks  SM clock and clock-event reasons sampled through NVML every 5 ms
        during the timed region.
Multi-GPU: independent replicas (one propagation per rank, weak scaling,
no data-path collective); rank times are reduced with MAX through the host
group of qd_b200.hostgroup.

--impl reference times the reference's own CPU propagator (common/timeEvol.C,
built in oracle/_ref against the shims) on the host cores for a bounded
sample of steps of the same workload.
"""
import argparse
import json
import os
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


def surrogate_c1(precision, n_train=400000, steps=240000, seed=12345, e_cut_ev=70.0):
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
    # trained over the whole capped range of the grid (2.5 hartree = 68 eV): the
    # packet's tails in the repulsive walls move P(E) (|dP| 0.015 with a 3 eV
    # training range, 0.0075 with 8 eV, 0.0047 with 70 eV, same network)
    r12, r23, r13, V = training_set(pes, m_amu, n=n_train, seed=seed, e_cut_ev=e_cut_ev)
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
            "training_range_eV": e_cut_ev,
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


class GpuClock:
    """SM clock and clock-event reasons of this process's GPU, sampled every
    `period` seconds by a thread through NVML (read-only queries) while the
    GPU phase of the benchmark runs; `mark` records the wall-clock bounds of
    the timed region, whose samples the summary uses (all samples of the
    phase when fewer than three fall inside it, which it then says)."""
    BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
            "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, local, period=0.005):
        self.local = local
        self.period = period
        self.samples = []          # (t, sm_mhz, reasons bitmask)
        self.marks = {}
        self.max_mhz = None
        self.nv = None
        self._stop = False

    def _handle(self, nv):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x.strip() for x in vis.split(",") if x.strip()] if vis else []
        if ids and self.local < len(ids):
            tok = ids[self.local]
            if tok.isdigit():
                return nv.nvmlDeviceGetHandleByIndex(int(tok))
            return nv.nvmlDeviceGetHandleByUUID(tok)
        return nv.nvmlDeviceGetHandleByIndex(self.local)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception as e:          # no NVML: the line says so
            self.error = str(e)
            self.nv = None
        return self

    def _run(self):
        nv = self.nv
        while not self._stop:
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def mark(self, name):
        self.marks[name] = time.perf_counter()

    def __exit__(self, *a):
        self._stop = True
        if self.nv:
            self.t.join(timeout=2)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "source": getattr(self, "error", "no samples")}
        t0, t1 = self.marks.get("timed_begin"), self.marks.get("timed_end")
        inside = [x for x in self.samples if t0 is not None and t1 is not None and t0 <= x[0] <= t1]
        use, window = (inside, "timed region") if len(inside) >= 3 else \
            (self.samples, "whole GPU phase (warm-up, timed, profiled and unflushed steps)")
        reasons = sorted(n for n, b in self.BITS.items() if any(x[2] & b for x in use))
        return {"sm_mhz": float(np.median([x[1] for x in use])), "sm_max_mhz": self.max_mhz,
                "sm_min_mhz": float(min(x[1] for x in use)), "reasons": reasons,
                "samples": len(use), "samples_timed_region": len(inside), "window": window,
                "source": f"NVML every {self.period * 1e3:.0f} ms"}


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


def group_setup():
    """Rank, world, local GPU and the host group of this process (one process
    per GPU, launched by torchrun or alone); the group gives the barrier and
    the max over ranks, with no device library involved."""
    from qd_b200.hostgroup import FileGroup
    g = FileGroup.from_env()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return g.rank, g.world, local, g


def run_reference(args):
    rank, world, local, grp = group_setup()
    if rank != 0:
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


KCLASS = ["column", "lines", "flux_prep", "flux_accum", "crp"]


def device_phase(data, prec, K, W, clk=None, profile=True):
    """Device-resident rate of one precision: W warm-up steps, then K timed
    steps (CUDA events on the library's stream, L2 flushed before every step
    outside the timed spans); then, untimed for the rate, a profiled run
    (per-kernel-class CUDA events), K plain steps (no per-step events, no
    flush: the library's own launch chain) and K unflushed timed steps."""
    from qd_b200 import Propagator
    from qd_b200 import _abi
    from qd_b200.timeevolution import kernel_launch_count
    import ctypes as C
    d = copy_workload(data)
    for r in as_runs(d):
        r.options.precision = prec
    out = {}
    with Propagator(d) as p:
        p.propagate_timed(W, FLUSH_BYTES)
        l0 = kernel_launch_count()
        if clk:
            clk.mark("timed_begin")
        out["ms"] = p.propagate_timed(K, FLUSH_BYTES)
        if clk:
            clk.mark("timed_end")
        out["launches"] = kernel_launch_count() - l0
        if profile:
            lib = _abi.lib()
            lib.qd_set_profiling(p._h, 1)
            p.propagate(min(K, 400))
            buf = (C.c_double * 10)()
            nw = C.c_int32()
            lib.qd_kernel_times(p._h, buf, 10, C.byref(nw))
            lib.qd_set_profiling(p._h, 0)
            kc = list(buf)[:nw.value]
            out["kclass_ms"] = {KCLASS[i]: kc[i] for i in range(min(5, len(kc)))}
            ch = (C.c_int32 * 4)()
            lib.qd_kernel_choice(p._h, ch)
            out["choice"] = list(ch)
            t0 = time.perf_counter()
            p.propagate(K)
            out["plain_s"] = time.perf_counter() - t0
            out["ms_warm"] = p.propagate_timed(K, 0)
    return out


SLICE_KINDS = {0: "split row and column kernels", 1: "Stockham cluster kernel, 1 CTA per slice",
               2: "Stockham cluster kernel, 2-CTA clusters", 4: "Stockham cluster kernel, 4-CTA clusters",
               8: "register-FFT kernel k_slice_rf, 1 CTA per slice",
               9: "register-FFT kernel k_slice_rf, 2-CTA clusters",
               10: "register-FFT kernel k_slice_rf, 4-CTA clusters",
               11: "register-FFT kernel k_slice_rf, 4-CTA clusters, 16x16 row transforms"}


def describe_choice(ch, fp64):
    """The autotuners' picks for the timed handle (qd_kernel_choice)."""
    return {"l_space": "FP64 split kernels" if fp64 else SLICE_KINDS.get(ch[0], str(ch[0])),
            "column": "tensor cores (k_column_tc, tcgen05 kind::f16)" if ch[1] else "SIMT",
            "flux_gemm_variant": ch[2],
            "flux_full_chunks": "chirp-z (k_flux_czt)" if ch[3] else "direct GEMM (k_flux_gemm)"}


def roofline_entry(name, alg_bytes, ms, peak, peak_kind, traffic):
    ach = alg_bytes / (ms * 1e-3) / 1e9 if ms and ms > 0 else None
    return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": ach / peak if ach else None,
            "traffic": traffic, "traffic_unit": "DRAM bytes read + written per launch (ncu)",
            "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": ms}


# DRAM bytes (read + write) per launch of the column and l-space kernels
# from one ncu capture each (cold caches: ncu flushes them before every
# captured launch); the batch figures were captured on fewer runs and scale
# with the runs (traffic_runs).  The ncu summaries under profiles/ give the
# commands that made them.
TRAFFIC_NCU = {("c1", "column"): (16.89e6, 1), ("c1", "lines"): (9.30e6, 1),
               ("c2j0", "column"): (373.7e6, 32), ("c2j0", "lines"): (379.7e6, 32),
               ("c4", "column"): (568.4e6, 4), ("c4", "lines"): (360.6e6, 4)}


def run_ours(args):
    rank, world, local, grp = group_setup()
    from qd_b200 import QD_PREC_FP32, QD_PREC_FP64, TimeEvolutionMexCUDA
    from qd_b200.timeevolution import set_device
    set_device(local)
    prec = QD_PREC_FP64 if args.fp64 else QD_PREC_FP32
    data, desc = build_workload(args.workload, prec, args.runs)
    runs = as_runs(data)
    pts = grid_points(data)
    K, W = args.steps, args.warmup

    # --- device-resident throughput, clocks sampled over the whole GPU phase ------------
    grp.barrier()
    with GpuClock(local) as clk:
        dev = device_phase(data, prec, K, W, clk)
    t_max = grp.max(dev["ms"])
    value = pts * K * world / (t_max * 1e-3)

    # --- the plain FP64 form on the same workload (the batched form's speed-up over it) ---
    fp64 = None
    if not args.fp64 and not args.no_fp64_arm:
        grp.barrier()
        d64 = device_phase(data, QD_PREC_FP64, K, W, profile=False)
        t64 = grp.max(d64["ms"])
        v64 = pts * K * world / (t64 * 1e-3)
        fp64 = {"value": v64, "unit": METRIC, "ms_per_step": t64 / K,
                "ratio": value / v64, "steps": K,
                "what": "the plain form (complex128 wavepacket, FP64 everywhere) on the same "
                        "workload and GPU, timed the same way"}

    # --- the same passes in their library forms (context for the FP64 ratio) -------------
    libform = None
    if not args.fp64 and not args.no_lib_compare and world == 1:
        lib = library_form(data, max(K, 5))
        ours_ms = dev["kclass_ms"].get("column", 0.0) + dev["kclass_ms"].get("lines", 0.0)
        lib64 = lib["column_cublas_fp64_ms"] + lib["lspace_cufft_z2z_ms"]
        lib32 = lib["column_cublas_fp32_bf16x9_ms"] + lib["lspace_cufft_c2c_ms"]
        libform = {**lib, "ours_column_plus_lspace_ms": ours_ms,
                   "library_fp64_column_plus_lspace_ms": lib64,
                   "library_fp32_column_plus_lspace_ms": lib32,
                   "ratio_vs_library_fp64": lib64 / ours_ms if ours_ms else None,
                   "ratio_vs_library_fp32": lib32 / ours_ms if ours_ms else None,
                   "what": "the column and l-space passes of one step: ours (complex64, per-kernel "
                           "CUDA events) against cuBLAS Legendre GEMMs + cuFFT 2-D plans + "
                           "elementwise phase kernels on the same shapes, FP64 (Z2Z, DGEMM) and "
                           "FP32 (C2C, BF16x9-emulated FP32 GEMM)"}

    # --- end to end through the drop-in entry point -------------------------------
    # each a full call: upload, set-up, K steps, P(E), download; median reported
    nrep = 5 if pts * 16 < (1 << 30) else 3
    reps = []
    for _ in range(nrep):
        e = copy_workload(data)
        for r in as_runs(e):
            r.time.total_steps = K
            r.time.steps = 0
        grp.barrier()
        t0 = time.perf_counter()
        TimeEvolutionMexCUDA(e)
        reps.append(time.perf_counter() - t0)
    e2e_s = grp.max(float(np.median(reps)))
    h2d = sum(r.pot.nbytes + r.psi.nbytes for r in runs) + runs[0].theta.legendre.nbytes
    d2h = sum(r.psi.nbytes + r.CRP.CRP.nbytes for r in runs)
    e2e = {"value": pts * K * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
           "seconds": e2e_s, "seconds_each": reps,
           "entry_point": f"qd_time_evolution (TimeEvolutionMexCUDA), median of {nrep} calls"}

    if rank != 0:
        return

    # --- roofline of the two hot kernels ------------------------------------------------
    peak, peak_kind = load_peaks()
    r0 = runs[0]
    nl, nth = int(r0.theta.m) + 1, int(r0.theta.n)
    nl = max(int(r.theta.m) + 1 for r in runs)
    n12 = int(r0.r1.n) * int(r0.r2.n) * len(runs)
    cb = 16 if args.fp64 else 8        # bytes per complex
    shared_pot = all(np.array_equal(r.pot, r0.pot) for r in runs[1:])
    npot = 1 if shared_pot else len(runs)
    alg = {  # algorithmic bytes per launch: psi_l read + written, exp(-iV dt) read once
        "column": n12 * 2 * nl * cb + int(r0.r1.n) * int(r0.r2.n) * nth * cb * npot,
        "lines": n12 * nl * 2 * cb,
    }
    per = dev.get("kclass_ms", {})
    kernels = {}
    for k in ("column", "lines"):
        tr = None
        if not args.fp64 and (args.workload, k) in TRAFFIC_NCU:
            b, nr = TRAFFIC_NCU[(args.workload, k)]
            tr = b * len(runs) / nr
        kernels[k] = roofline_entry(k, alg[k], per.get(k), peak, peak_kind, tr)
    dom = max(("column", "lines"), key=lambda k: per.get(k, 0.0))
    roofline = dict(kernels[dom])
    roofline["kernels"] = {k: {x: kernels[k][x] for x in ("achieved", "frac", "avg_launch_ms",
                                                          "alg_bytes_per_launch", "traffic")}
                           for k in kernels}
    roofline["kernel_class_ms"] = per
    if dev.get("choice"):
        roofline["tuned"] = describe_choice(dev["choice"], args.fp64)
    step_ms = t_max / K
    step_bytes = 36 if not args.fp64 else 72
    roofline["whole_step"] = {"alg_bytes_per_grid_pt_step": step_bytes,
                              "achieved": pts * step_bytes / (step_ms * 1e-3) / 1e9,
                              "frac": pts * step_bytes / (step_ms * 1e-3) / 1e9 / peak}

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
                       "complex64 + 3xFP16 Legendre + FP64 flux accumulation",
                       "l2": "flushed before every step (256 MiB written, then read back so "
                             "no dirty lines remain; outside the timed spans)",
                       "parallelism": f"replicas x{world}"},
            "value_l2_resident": pts * K / (dev["ms_warm"] * 1e-3),
            "value_plain_call": pts * K / dev["plain_s"],
            "fp64_plain": fp64, "library_form": libform,
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clk.summary(), "gpu_launches": dev["launches"], **EXTRA,
            "pe_curves_per_hour_e2e": curves_per_hour}
    print(json.dumps(line))


def library_form(data, reps):
    """ms per step of the column and l-space passes in their library forms
    (cuFFT plans, cuBLAS GEMMs, elementwise phase kernels) on the workload's
    shapes, from lib/libqd_libcmp.so."""
    from qd_b200 import libcompare as LC
    LC.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    runs = as_runs(data)
    r0 = runs[0]
    n1, n2, nth = int(r0.r1.n), int(r0.r2.n), int(r0.theta.n)
    nl = max(int(r.theta.m) + 1 for r in runs)
    lib = {"lspace_cufft_c2c_ms": LC.lspace_cufft_ms(n1, n2, nl, len(runs), False, reps),
           "lspace_cufft_z2z_ms": LC.lspace_cufft_ms(n1, n2, nl, len(runs), True, reps)}
    for c in LC.COMPUTE:
        lib[f"column_cublas_{c}_ms"] = LC.column_cublas_ms(n1, n2, nth, nl, len(runs), c, reps)
    return lib


def run_compare_libs(args):
    """This library's column and l-space passes against the same passes on
    cuFFT and cuBLAS (the reference GPU code's design), per step of the
    workload, on one GPU.  Prints one JSON line."""
    from qd_b200 import QD_PREC_FP32, QD_PREC_FP64
    from qd_b200 import libcompare as LC
    from qd_b200.timeevolution import set_device
    set_device(0)
    LC.set_device(0)
    data, desc = build_workload(args.workload, QD_PREC_FP32, args.runs)
    runs = as_runs(data)
    r0 = runs[0]
    n1, n2, nth = int(r0.r1.n), int(r0.r2.n), int(r0.theta.n)
    nl = max(int(r.theta.m) + 1 for r in runs)
    K = max(args.steps, 10)
    ours = {}
    for name, prec in (("complex64", QD_PREC_FP32), ("fp64", QD_PREC_FP64)):
        dev = device_phase(data, prec, K, 3)
        ours[name] = {"column_ms": dev["kclass_ms"]["column"],
                      "lspace_ms": dev["kclass_ms"]["lines"], "step_ms": dev["ms"] / K}
    lib = library_form(data, K)
    c64, f64 = ours["complex64"], ours["fp64"]
    ratios = {
        "lspace_complex64": lib["lspace_cufft_c2c_ms"] / c64["lspace_ms"],
        "lspace_fp64": lib["lspace_cufft_z2z_ms"] / f64["lspace_ms"],
        "column_complex64_vs_fp32_bf16x9": lib["column_cublas_fp32_bf16x9_ms"] / c64["column_ms"],
        "column_complex64_vs_fp32_simt": lib["column_cublas_fp32_simt_ms"] / c64["column_ms"],
        "column_complex64_vs_tf32": lib["column_cublas_tf32_ms"] / c64["column_ms"],
        "column_fp64": lib["column_cublas_fp64_ms"] / f64["column_ms"],
    }
    print(json.dumps({"compare_libs": {"workload": desc, "steps": K, "ours": ours,
                                       "library": lib, "library_over_ours": ratios,
                                       "note": "library forms: one batched cufftPlanMany 2-D "
                                               "transform pair with the phases as elementwise "
                                               "kernels; strided-batched cublasGemmEx Legendre "
                                               "pair with the potential phase elementwise; ours: "
                                               "per-kernel-class CUDA events of the propagator"}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c1", "c0", "c2", "c2j0", "c3", "c4"])
    ap.add_argument("--runs", type=int, default=64, help="runs of the c2j0 batch")
    ap.add_argument("--fp64", action="store_true", help="plain FP64 form instead of complex64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="skip the plain FP64 form's rate on the same workload")
    ap.add_argument("--no-lib-compare", action="store_true",
                    help="skip the library forms of the passes in the default line")
    ap.add_argument("--compare-libs", action="store_true",
                    help="time the column and l-space passes against cuBLAS / cuFFT forms")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.compare_libs:
        run_compare_libs(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
