"""Benchmark: converged AC power-flow solves/s on one B200.

Workload (one "step"): the full N-1 contingency sweep of the seeded synthetic
2000-bus grid (3200 branches, 400 PV buses, 1500 loads): every single-branch
outage that keeps the grid connected (2847 rows for seed 0), ||F||inf < 1e-8
pu, at most 10 Newton steps per row, one symbolic analysis shared by every
row.  Default arm (``--start learned``): each row starts from the voltages
the warm-start MLP predicts for it (features -> BF16 MLP on tcgen05 -> V0,
on the device), then the mixed-precision sweep converges it; the network is
trained before the run (untimed, reported under ``training``) on 100k
GPU-solved synthetic operating points.  The comparison arm is the same rows
solved by plain FP64 Newton from a flat start (``fp64_flat_value``).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--start learned|flat] [--precision mixed|fp64]

`value`  : rows converged per second; device time per step = CUDA events
           around features + MLP + V0 (torch's stream) + the sweep kernel
           (CUDA events on the session stream); inputs resident in HBM; L2
           flushed (256 MiB write) before every timed step.
`e2e`    : the same metric through the public facade with host buffers
           (contingency lists in, voltages + statuses + residuals out).
`cfg2`   : (default workload only) the 6500-bus injection sweep measured the
           same way: value, FP64 comparison, agreement, roofline.
`cpu_baseline` / --impl reference: the compiled CPU restatement of the
           reference's Newton-Raphson (oracle/cpu_nr.cpp: FP64, own sparse LU,
           OpenMP over rows on every host thread) over all rows of the same
           workload, or a sample sized to --cpu-budget-s when they take longer.
With N > 1 (torchrun), every rank solves its own copy of the workload
(replicas: rows are independent, there is no collective on the data path);
time is the max over ranks.
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# name -> (grid, row kind, rows, scenario seed, training-row mix)
WORKLOADS = {
    # one system solved again and again (the single-solve path, AcPfGPU / acpf_nr_gpu), 118-bus grid
    "single_case118_synth": ("case118_synth", "single", 1, None, {}),
    # every non-islanding single outage of the 2000-bus grid at base injections
    "n1_sweep_case2000_synth": ("case2000_synth", "n1", None, None, dict(broad=0.5)),
    # 4096 load-scaling scenarios (global U(0.8,1.2) x per-bus lognormal(0,0.1)) on the 6500-bus grid
    "injection_sweep_case6500_synth": ("case6500_synth", "injection", 4096, 1, dict(broad=1.0, p_outage=0.0)),
    # 16384 rows on the 2000-bus grid, each a load-scaling scenario plus one single outage
    "injection_n1_case2000_synth": ("case2000_synth", "injection_n1", 16384, 1, dict(broad=1.0, p_outage=0.9)),
    # 8192 rows, 2048 on each of the 118/2000/6500/10000-bus grids, each a load-scaling scenario plus 0-2
    # tripped non-islanding branches, all in one persistent launch
    "heterogeneous_8192_case118_2000_6500_10000": ("case118_synth,case2000_synth,case6500_synth,case10000_synth",
                                                    "multi", 2048, 3, dict(broad=1.0, p_outage=0.9)),
}
MAX_ITER, TOL = 10, 1e-8
LOAD_SCALE = 1.0  # --load-scale: heavier (or lighter) loading of every grid
METRIC = "Converged AC PF solves/s on 1 B200: learned+mixed vs plain FP64 NR @1e-8 pu"

def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--strategy", choices=["auto", "adaptive", "base_chord", "refactor_every"], default="auto",
                    help="linear-solve strategy of the measured arm (the FP64 comparison arm always refactors); "
                         "auto: base_chord (rows chord on the base case's factor, outages by Woodbury compensation)")
    ap.add_argument("--refactor-ratio", type=float, default=None,
                    help="contraction ratio above which a row factors its own Jacobian (default: the facade's)")
    ap.add_argument("--max-reuse", type=int, default=None, help="chord steps on one factor at most (default: the facade's)")
    ap.add_argument("--cpu-budget-s", type=float, default=8.0,
                    help="seconds one CPU-baseline pass may take: all rows if they fit, else a sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows", type=int, default=0, help="solve only the first ROWS rows (profiling cases)")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="n1_sweep_case2000_synth")
    ap.add_argument("--start", choices=["learned", "flat"], default="learned",
                    help="learned: MLP warm start (trained untimed before the run); flat: Vinit")
    ap.add_argument("--train-rows", type=int, default=100000)
    ap.add_argument("--cfg2-steps", type=int, default=10,
                    help="timed steps of the 6500-bus injection sweep carried in the default line's cfg2 object "
                         "(0: leave it out)")
    ap.add_argument("--cfg2-train-rows", type=int, default=20000)
    ap.add_argument("--train-epochs", type=int, default=20)
    ap.add_argument("--load-scale", type=float, default=1.0,
                    help="multiply every grid's loads (and the generation following them): the strategy under "
                         "heavier loading (1.0: the configs' grids)")
    ap.add_argument("--hidden", type=int, default=1024)
    ap.add_argument("--tune-rates", type=float, nargs="*", default=[40.0, 160.0, 320.0],
                    help="dense/scatter cost ratios the plan autotuner tries (none: keep the default plan)")
    return ap.parse_args()


def _dist():
    """(rank, world size, local rank) from torchrun's environment (1 process
    without it).  Read here rather than through the package, so that the
    reference arm never loads this repository's native library."""
    env = os.environ
    return int(env.get("RANK", 0)), int(env.get("WORLD_SIZE", 1)), int(env.get("LOCAL_RANK", 0))


_SYNTH = None


def _synthetic():
    """gpusim2grid_b200/synthetic.py loaded by its path: the grid generator is
    plain numpy, and importing it through the package would load the native
    library (the reference arm must run without it)."""
    global _SYNTH
    if _SYNTH is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("gs2g_bench_synthetic",
                                                      os.path.join(ROOT, "gpusim2grid_b200", "synthetic.py"))
        _SYNTH = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = _SYNTH  # dataclasses resolves the module by name
        spec.loader.exec_module(_SYNTH)
    return _SYNTH


def _native_maps():
    """This process's mapped shared objects that belong to this repository's
    engine (the reference arm must show none)."""
    try:
        with open("/proc/self/maps") as fh:
            paths = {ln.split()[-1] for ln in fh if ln.rstrip().endswith(".so") or ".so." in ln}
    except OSError:
        return None
    return sorted(p for p in paths if "gs2g" in os.path.basename(p))


def _workload(name):
    """(grid, trips or None, p_mw or None, q_mvar or None) of a named workload;
    for the heterogeneous workload, a list of such tuples (one per grid)."""
    syn = _synthetic()
    injection_scenarios = syn.injection_scenarios

    def grid_by_name(name, seed):
        # the configs' grid, its loads (and the generation following them)
        # times --load-scale
        n_bus, n_branch, n_pv, n_load, n_trafo, scale = syn.GRID_SPECS[name]
        return syn.make_grid(n_bus, n_branch, n_pv, n_load, n_trafo, seed=seed, name=name,
                             load_scale=scale * LOAD_SCALE)
    n1_branches, scenario_outages = syn.n1_branches, syn.scenario_outages
    gname, kind, n_rows, seed, _ = WORKLOADS[name]
    if kind == "multi":
        parts = []
        for i, gn in enumerate(gname.split(",")):
            g = grid_by_name(gn, 0)
            p, q = injection_scenarios(g, n_rows, seed=seed + 10 * i)
            parts.append((g, scenario_outages(g, n_rows, max_trips=2, seed=seed + 10 * i + 1), p, q))
        return parts
    g = grid_by_name(gname, 0)
    if kind == "single":
        return g, None, None, None
    cand = n1_branches(g)
    if kind == "n1":
        return g, [[int(b)] for b in cand], None, None
    p, q = injection_scenarios(g, n_rows, seed=seed)
    if kind == "injection":
        return g, None, p, q
    return g, [[int(cand[r % cand.size])] for r in range(n_rows)], p, q


# ---------------------------------------------------------------- CPU side
def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.lower().startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


class CpuBaseline:
    """The compiled CPU Newton-Raphson (oracle/cpu_nr.cpp: FP64, flat start,
    own minimum-degree ordering, static-pivot sparse + dense LU refactored
    every step, OpenMP over rows on every host thread) over a workload's
    rows: all of them when a calibration pass says they fit ``budget_s``,
    else an evenly spaced sample sized to it."""

    def __init__(self, g, trips, p, q, budget_s=8.0):
        from oracle import cpu_nr
        self.cpu_nr = cpu_nr
        self.g, self.trips, self.p, self.q = g, trips, p, q
        self.n = len(trips) if trips is not None else p.shape[0]
        self.threads = _host_threads()
        cal = np.unique(np.linspace(0, self.n - 1, min(self.n, 2 * self.threads)).astype(int))
        _, dt = self._run(cal)
        rate = len(cal) / dt
        k = self.n if self.n / rate <= budget_s else max(len(cal), int(rate * budget_s))
        self.idx = np.arange(self.n) if k >= self.n else np.unique(np.linspace(0, self.n - 1, k).astype(int))
        self.sample = (f"{len(self.idx)} of {self.n} rows" + (" (all)" if len(self.idx) == self.n else
                                                               " (evenly spaced)")
                       + ", flat start, compiled FP64 NR (oracle/cpu_nr.cpp), OpenMP over rows")

    def _run(self, idx):
        g = self.g
        Y, V0, S, _, _, pv, pq = g.as_tuple()
        t = [self.trips[r] for r in idx] if self.trips is not None else None
        sb = None if self.p is None else (self.p[idx] + 1j * self.q[idx]) / g.sn_mva
        br = (g.branch_from, g.branch_to, g.yff, g.yft, g.ytf, g.ytt) if t is not None else None
        t0 = time.perf_counter()
        _, st, _, _, _ = self.cpu_nr.sweep(Y, V0, S, pv, pq, branches=br, trips=t, sbus_rows=sb, max_iter=MAX_ITER,
                                           tol=TOL, threads=self.threads)
        return int((st == 0).sum()), time.perf_counter() - t0

    def measure(self):
        """Converged solves/s of one pass over the chosen rows."""
        conv, dt = self._run(self.idx)
        return conv / dt


def cpu_baseline(g, trips, p, q, budget_s=8.0):
    """(solves/s, threads, sample description) of one timed pass."""
    cb = CpuBaseline(g, trips, p, q, budget_s)
    return cb.measure(), cb.threads, cb.sample


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, max clock and clock-event reasons of the bench's GPU during
    the timed region (read-only queries).  NVML every 10 ms when the bindings
    load -- the device found by its PCI bus id, so CUDA_VISIBLE_DEVICES does
    not shift it -- else nvidia-smi every 0.2 s."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            self._nvml = (pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus))
        except Exception:
            self._nvml = None

    def start(self):
        self._t = threading.Thread(target=self._run_nvml if self._nvml else self._run, daemon=True)
        self._t.start()

    def _run_nvml(self):
        while not self._stop.is_set():
            self._sample_nvml()
            self._stop.wait(0.01)

    def _sample_nvml(self):
        nv, h = self._nvml
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        try:
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append([str(self.index), str(sm), str(mx), "",
                                 *["Active" if r & b else "Not Active" for b in bits]])
        except Exception:
            pass

    def _run(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                r = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if r.returncode == 0 and r.stdout.strip():
                    self.samples.append([x.strip() for x in r.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples and self._nvml:
            # a timed region shorter than the first poll: one reading at its end
            self._sample_nvml()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if "Active" in s[4 + i]
                          and "Not" not in s[4 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


AGREE_PU = 1e-6  # the metric's agreement bar with the FP64 flat-start answer


def _counted(V, st, V64, st64):
    """Rows that count for the metric: converged here and in plain FP64 NR
    from flat, to the same solution (max |dV| <= AGREE_PU)."""
    ok = (np.asarray(st) == 0) & (np.asarray(st64) == 0)
    if not ok.any():
        return 0
    dv = np.abs(np.asarray(V)[ok] - np.asarray(V64)[ok]).max(axis=1)
    return int((dv <= AGREE_PU).sum())


def algorithmic_bytes(info, w):
    """Minimum bytes (shared structure amortised to zero) of one LU
    factorization of one row (J write and read, factor write) and of one
    Newton step of one row (V read, outage edits, F write, factor read by the
    solves, rhs/x, dx read, V read-modify-write).  w = 8 (FP64) or 4 (FP32)."""
    n, d, nJ, nLU = info["n_bus"], info["dim_j"], info["nnz_j"], info["nnz_lu"]
    per_factor = w * nJ * 2 + w * nLU
    per_iter = 16 * n + 16 * 4 + 8 * d + w * nLU + 16 * d + 8 * d + 32 * n
    return per_factor, per_iter


def algorithmic_flops(info):
    """FLOPs of one LU factorization (2 per madd) and of one Newton step
    (two triangular solves + SpMV/Jacobian complex arithmetic)."""
    lu = info["head_madds"] + info["schur_madds"] + info["dense_madds"]
    return 2 * lu, 4 * info["nnz_lu"] + 40 * info["nnz_y"]


# ---------------------------------------------------------------- our arm
def _train_learned(g, args, device, workload, n_rows=None):
    from gpusim2grid_b200.warmstart import LearnedStart
    ls = LearnedStart(g, hidden=args.hidden, layers=2, device=device, seed=0)
    mix = dict(WORKLOADS[workload][4])
    rep = ls.train(n_rows=args.train_rows if n_rows is None else n_rows, epochs=args.train_epochs, batch=1024,
                   lr=1e-3, lr_decay=0.8, seed=7, **mix)
    return ls, rep, mix


def _strategy(args, trips):
    if args.strategy != "auto":
        return args.strategy
    return "base_chord"


def _facade(g, trips, p, q, args, local):
    """The reference-facing facade for the workload's rows (host inputs)."""
    from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, ScenarioSweepGPU
    kw = dict(init_from_n_powerflow=False, precision=args.precision, nb_iter=MAX_ITER, scheduling="continuous",
              tol=TOL, start="flat", device=local, strategy=_strategy(args, trips))
    if p is None:
        f = ContingencyAnalysisGPU(g.as_tuple(), **kw)
        f.set_branch_data(*g.branch_data())
        f.add_contingencies_by_branch_id(trips)
    elif trips is None:
        f = InjectionSweepGPU(g.as_tuple(), **kw)
        f.set_injections(p, q, g.sn_mva)
    else:
        f = ScenarioSweepGPU(g.as_tuple(), **kw)
        f.set_branch_data(*g.branch_data())
        f.set_injections(p, q, g.sn_mva)
        f.set_topology(trips)
    return f


def _set_rows(f, trips, p, q, g):
    """Hand the workload's host row definitions to the facade again (e2e)."""
    if p is None:
        f.add_contingencies_by_branch_id(trips)
    elif trips is None:
        f.set_injections(p, q, g.sn_mva)
    else:
        f.set_injections(p, q, g.sn_mva)
        f.set_topology(trips)


def measure(args, workload, steps, warmup, train_rows, rows_limit=0, e2e=True):
    """One single-grid workload on this rank's GPU: the measured arm (timed
    device steps), the comparison arms on the same rows, the roofline inputs
    and, with e2e, the same metric through the facade with host buffers.
    Returns (line dict, workload tuple)."""
    import torch
    from gpusim2grid_b200 import RowStatus, replicas
    from gpusim2grid_b200._native import lib
    _, world, local = _dist()

    g, trips, p, q = _workload(workload)
    if rows_limit > 0:
        trips = trips[:rows_limit] if trips is not None else None
        p, q = (p[:rows_limit], q[:rows_limit]) if p is not None else (None, None)
    n = len(trips) if trips is not None else p.shape[0]
    learned = args.start == "learned"
    prec = lib.PREC_MIXED if args.precision == "mixed" else lib.PREC_FP64
    ca = _facade(g, trips, p, q, args, local)
    strat = {"adaptive": lib.REFACTOR_ADAPTIVE, "base_chord": lib.REFACTOR_BASE_CHORD,
             "refactor_every": lib.REFACTOR_EVERY}[_strategy(args, trips)]
    s = ca.session
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # device-resident row definitions for the learned start's features
    csr = _ids(trips) if trips is not None else None
    sbus_dev = None if p is None else torch.as_tensor((p + 1j * q) / g.sn_mva, device="cuda")

    train = None
    ls = None
    ratio, reuse = 0.0, 0
    if learned:
        t0 = time.perf_counter()
        ls, rep, mix = _train_learned(g, args, local, workload, n_rows=train_rows)
        train = {"rows": rep["n_rows"], "epochs": args.train_epochs, "hidden": args.hidden, "layers": 2,
                 "row_mix": mix, "unconverged_dropped": rep["n_unconverged"],
                 "t_generate_solve_s": round(rep["t_rows_s"] + rep["t_solve_s"], 2),
                 "t_fit_s": round(rep["t_fit_s"], 2), "t_total_s": round(time.perf_counter() - t0, 2),
                 "loss_first_last": [round(rep["loss"][0], 5), round(rep["loss"][-1], 5)],
                 "val_mse": round(rep["val"][-1], 5) if rep["val"] else None,
                 "note": "untimed: training rows are seeded synthetic operating points (load scaling, single "
                         "outages) solved by this engine in FP64, drawn with another seed than the timed rows"}
        ca.set_learned_start(ls, args.refactor_ratio, args.max_reuse)
        ratio, reuse = ca._learned_opts
    elif strat == lib.REFACTOR_BASE_CHORD:
        ratio, reuse = 0.7, 8
    # one-time plan choice (untimed, like the symbolic analysis): the
    # head/tail split that solves these rows fastest in the measured arm
    ca.start = "learned" if learned else "flat"
    tune, rate = ca.autotune(tuple(args.tune_rates), repeats=1) if args.tune_rates else ({}, None)
    info = s.info()
    start_mode = lib.START_ROWS if learned else lib.START_VINIT
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def step():
        """Device ms of one pass: [features -> MLP -> V0 (torch's stream)] + sweep kernel (session stream)."""
        pre_ms = 0.0
        if learned:
            buf = s.start_rows_buffer(n)
            ev0.record()
            ls.start_voltages(sbus_dev, csr, n, out_ptr=buf)
            ev1.record()
            ev1.synchronize()
            pre_ms = ev0.elapsed_time(ev1)
        s.run(MAX_ITER, TOL, False, prec, start_mode, 0.0, 0, False, strat, ratio, reuse, learned)
        tm = s.timings()
        ms = tm["kernel_ms"]
        sweep_log.append((ms, int(tm["chord_steps"])))
        # rows left unconverged are re-solved in plain FP64 (part of the timed work)
        return pre_ms, ms + ca.fp64_fallback()

    sweep_log = []  # (sweep-launch ms, Newton steps on the shared base factor) per step
    for _ in range(warmup):
        step()
    setup = {"base_factor_ms": round(float(s.timings()["base_setup_ms"]), 2),
             "base_factor_bytes": int(s.timings()["base_setup_bytes"]),
             "note": "once per session, base case and precision (the shared base factor, its explicit inverse and "
                     "solve-ordered values), untimed like the symbolic analysis"} \
        if strat == lib.REFACTOR_BASE_CHORD else None
    clk = ClockSampler(local)
    clk.start()
    replicas.barrier()
    pre, ker = [], []
    torch.cuda.nvtx.range_push("bench_timed")  # ncu --nvtx --nvtx-include bench_timed/
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a_, b_ = step()
        pre.append(a_)
        ker.append(b_)
    torch.cuda.nvtx.range_pop()
    replicas.barrier()
    clocks = clk.stop()
    total_ms = replicas.max_over_ranks(float(np.sum(pre) + np.sum(ker)), device="cuda")
    fallback_rows = ca.fallback_rows
    V_w, res, st, it = s.results()
    n_conv = int((st == RowStatus.CONVERGED).sum())
    total_iters = int(it.sum())
    total_factors = int(s.factor_counts().sum())
    n_rescued = int(s.timings()["n_rescued"])
    value = world * n_conv * steps / (total_ms / 1e3)
    iters_hist = {int(k): int(v) for k, v in zip(*np.unique(it, return_counts=True))}

    # comparison arms on the same rows (device time of the sweep, L2 flushed)
    def arm(p_, strat_, start_, ratio_=0.0, reuse_=0):
        s.run(MAX_ITER, TOL, False, p_, start_, 0.0, 0, False, strat_, ratio_, reuse_)
        ms_ = []
        for _ in range(max(1, min(steps, 3))):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            s.run(MAX_ITER, TOL, False, p_, start_, 0.0, 0, False, strat_, ratio_, reuse_)
            ms_.append(s.timings()["kernel_ms"])
        V_, _, st_, it_ = s.results()
        return int((st_ == 0).sum()) / (np.mean(ms_) / 1e3), V_, st_, it_

    # plain FP64 NR from flat: the metric's denominator
    fp64_value, V64, st64, it64 = arm(lib.PREC_FP64, lib.REFACTOR_EVERY, lib.START_VINIT)
    ok = (st == 0) & (st64 == 0)
    agree = float(np.abs(V_w[ok] - V64[ok]).max()) if ok.any() else None
    same_flags = bool(np.array_equal(st == 0, st64 == 0))
    # the metric counts a row when it converged here and in plain FP64 from
    # flat, to the same solution (|dV| <= 1e-6 pu)
    n_counted = _counted(V_w, st, V64, st64)
    value = world * n_counted * steps / (total_ms / 1e3)
    mixed_flat_value = base_start = None
    if learned and args.precision == "mixed":
        # mixed precision from flat (separates the strategy from the start)
        mixed_flat_value, _, _, _ = arm(lib.PREC_MIXED, lib.REFACTOR_ADAPTIVE, lib.START_VINIT)
        if strat == lib.REFACTOR_BASE_CHORD:
            # the same step from the base case's V without the network (sweep
            # and FP64 re-solve of the rows left unconverged): what the
            # learned start adds over the method without it
            def base_step():
                s.run(MAX_ITER, TOL, False, lib.PREC_MIXED, lib.START_BASE, 0.0, 0, False, strat, ratio, reuse)
                return s.timings()["kernel_ms"] + ca.fp64_fallback()

            base_step()
            ms_b = []
            for _ in range(max(1, min(steps, 3))):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                ms_b.append(base_step())
            Vb_, _, stb, itb = s.results()
            bv = _counted(Vb_, stb, V64, st64) / (np.mean(ms_b) / 1e3)
            base_start = {"value": round(bv, 1), "newton_iters_total": int(itb.sum()),
                          "rows_converged": int((stb == 0).sum()), "rows_fp64_fallback": ca.fallback_rows,
                          "learned_over_base_start": round(value / world / bv, 3),
                          "note": "same rows, precision and strategy, every row starting from the converged base "
                                  "case: the sweep and the FP64 re-solve of unconverged rows, without the network"}

    # phase split of the measured arm (one extra profiled run, not timed)
    if learned:
        ls.start_voltages(sbus_dev, csr, n, out_ptr=s.start_rows_buffer(n))
        torch.cuda.synchronize()
    s.run(MAX_ITER, TOL, False, prec, start_mode, 0.0, 0, True, strat, ratio, reuse, learned)
    phases = dict(zip(["mismatch", "fill", "head_lu", "schur", "dense_lu", "solve_head_fw", "solve_tail_fw",
                       "solve_dense", "solve_head_bw", "update"],
                      [round(x, 4) for x in s.timings()["phase_share"]]))

    e2e_obj = None
    if e2e:
        # end to end through the facade, host buffers in and out
        ca.start = "learned" if learned else "flat"
        # the kernels write each row's V into the page-locked result buffer
        # as the row leaves (the copy of V overlaps the sweep)
        ca.results_to_host = True
        # as a serving loop does after start-up: collect once and move the
        # start-up objects out of the collector's generations, so that a
        # full collection inside the loop scans only the loop's own objects
        gc.collect()
        gc.freeze()
        e2e_s, e2e_parts = [], []
        for i in range(warmup + steps):
            if i == warmup:
                e2e_s, e2e_parts = [], []
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _set_rows(ca, trips, p, q, g)
            t1 = time.perf_counter()
            ca.compute()
            t2 = time.perf_counter()
            # statuses, residuals and iterations into the same page-locked
            # buffer (one DMA each; V is already there)
            V, r, stt, itv = ca.results_view()
            t3 = time.perf_counter()
            e2e_s.append(t3 - t0)
            e2e_parts.append((t1 - t0, t2 - t1, t3 - t2, ca.timings.t_kernel_ms / 1e3))
        gc.unfreeze()
        e2e_value = world * _counted(V, stt, V64, st64) / float(np.mean(e2e_s))
        e2e_split = dict(zip(["rows_in_ms", "compute_ms", "results_out_ms", "kernel_ms"],
                             [round(float(x) * 1e3, 2) for x in np.mean(np.array(e2e_parts), axis=0)]))
        n_ids = sum(len(r_) for r_ in trips) if trips is not None else 0
        h2d = (4 * (n + 1) + 4 * n_ids if trips is not None else 0) + (2 * p.nbytes if p is not None else 0)
        d2h = V.nbytes + stt.nbytes + r.nbytes + itv.nbytes
        e2e_obj = {"value": round(e2e_value, 1), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "split": e2e_split}

    w = 4 if args.precision == "mixed" else 8
    b_fact, b_iter = algorithmic_bytes(info, w)
    if p is not None:
        b_iter += 16 * info["n_bus"]  # each step reads the row's Sbus
    # a step on the shared base factor reads no factor of its own: that
    # factor is shared structure, amortised to zero like the plan
    b_iter_shared = b_iter - w * info["nnz_lu"]
    chord_steps = sweep_log[-1][1]
    launch_bytes = b_fact * total_factors + b_iter_shared * chord_steps + b_iter * (total_iters - chord_steps)
    kernel_ms = float(np.mean([x[0] for x in sweep_log[-steps:]]))
    achieved_gbs = launch_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()
    f_fact, f_iter = algorithmic_flops(info)
    launch_flops = f_fact * total_factors + f_iter * total_iters
    achieved_tflops = launch_flops / (kernel_ms / 1e3) / 1e12
    fma_peak = 71.4 if args.precision == "mixed" else 37.1
    # base_chord: the chord sweep (after the outage-compensation setup of
    # rows that trip branches), then the single-row sweep for its hand-offs
    has_trips = WORKLOADS[workload][1] in ("n1", "injection_n1")
    sweep_launches = (3 if has_trips else 2) if strat == lib.REFACTOR_BASE_CHORD else 1
    per_step_launches = sweep_launches + (ls.launches_per_call(n, sbus_rows=WORKLOADS[workload][1] != "n1")
                                          if learned else 0) + (1 if fallback_rows else 0)
    gname = WORKLOADS[workload][0]

    line = {
        "metric": METRIC,
        "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": round(total_ms / steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 mismatch/V, f32 J/LU, bf16 MLP" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": workload, "grid": gname, "rows": n, "start": args.start,
                   "precision": args.precision, "strategy": _strategy(args, trips), "tol_pu": TOL, "max_iter": MAX_ITER,
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{world}",
                   "load_scale": LOAD_SCALE},
        "rows_converged": n_conv, "rows_counted": n_counted, "rows_rescued": n_rescued,
        "rows_fp64_fallback": fallback_rows,
        "newton_iters_total": total_iters,
        "lu_factorizations_total": total_factors, "mean_iters": round(total_iters / max(n, 1), 3),
        "iters_hist": iters_hist,
        "ms_split": {"features_mlp_v0": round(float(np.mean(pre)), 4), "sweep_kernel": round(kernel_ms, 4)},
        "fp64_flat_value": round(fp64_value, 1),
        "speedup_vs_fp64_flat": round(value / world / fp64_value, 3),
        "fp64_flat_iters_hist": {int(k): int(v) for k, v in zip(*np.unique(it64, return_counts=True))},
        "mixed_flat_value": None if mixed_flat_value is None else round(mixed_flat_value, 1),
        "base_start_value": base_start,
        "agreement_with_fp64": {"max_abs_dv_pu": agree, "rows_compared": int(ok.sum()),
                                "same_convergence_flags": same_flags},
        "training": train,
        "setup": setup,
        "plan": {"tail_dim": info["tail_dim"], "head_dim": info["head_dim"], "autotune_dense_rate": rate,
                 "autotune_ms": {str(k): v[1] for k, v in tune.items()}},
        "phase_share": phases,
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 4), "traffic": None,
                     "note": f"sweep launches of one step ({sweep_launches}); peak {peak_kind}; algorithmic bytes = "
                             f"{b_fact} per LU x {total_factors} LUs + {b_iter_shared} per step on the shared base "
                             f"factor x {chord_steps} + {b_iter} per step on a row's own factor x "
                             f"{total_iters - chord_steps}; the shared factor is served from L2, so the sweep is "
                             f"bound by L2 latency and bandwidth rather than HBM; DRAM traffic is measured by an "
                             f"ncu capture, not in this run"},
        "fma_roofline": {"achieved": round(achieved_tflops, 3), "peak": fma_peak, "unit": "TFLOP/s",
                         "frac": round(achieved_tflops / fma_peak, 4),
                         "note": "FP64 (or FP32) FMA pipe; peak measured by a DFMA/FFMA loop on this pool"},
        "e2e": e2e_obj,
        "gpu_launches": steps * per_step_launches,
        "clocks": clocks,
    }
    return line, (g, trips, p, q)


# the second workload of the default line: the 6500-bus injection sweep
# (its speed-up over plain FP64 is reported beside the N-1 sweep's)
CFG2 = "injection_sweep_case6500_synth"
CFG2_KEYS = ("value", "ms_per_step", "rows_converged", "rows_counted", "newton_iters_total", "lu_factorizations_total",
             "rows_fp64_fallback", "ms_split", "fp64_flat_value", "speedup_vs_fp64_flat", "mixed_flat_value",
             "base_start_value", "agreement_with_fp64", "training", "setup", "plan", "roofline", "clocks")


def run_ours(args):
    import torch
    from gpusim2grid_b200 import replicas
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=900)
    line, (g, trips, p, q) = measure(args, args.workload, args.steps, args.warmup, args.train_rows, args.rows)
    if args.workload == "n1_sweep_case2000_synth" and args.rows == 0 and args.cfg2_steps > 0:
        sub, _ = measure(args, CFG2, args.cfg2_steps, min(args.warmup, 3), args.cfg2_train_rows, e2e=False)
        line["cfg2"] = dict({"workload": CFG2, "rows": sub["config"]["rows"], "steps": sub["steps"]},
                            **{k: sub[k] for k in CFG2_KEYS})
        line["gpu_launches"] += sub["gpu_launches"]
    if rank == 0 and not args.no_cpu_baseline:
        v, cores, sample = cpu_baseline(g, trips, p, q, args.cpu_budget_s)
        line["cpu_baseline"] = {"value": round(v, 2), "unit": "solves/s", "cores": cores, "kind": "port",
                                "sample": sample, "cpu_model": _cpu_model()}
    replicas.finish()
    if rank == 0:
        print(json.dumps(line))


def _ids(rows):
    ptr = np.zeros(len(rows) + 1, dtype=np.int32)
    ptr[1:] = np.cumsum([len(r) for r in rows])
    return ptr, np.fromiter((b for r in rows for b in r), dtype=np.int32, count=int(ptr[-1]))


def cpu_baseline_multi(parts, budget_s=8.0):
    """The compiled CPU NR over every grid's rows (an equal share of the time
    budget each); the workload holds equal row counts per grid, so its rate
    is the harmonic mean of the per-grid rates."""
    secs, cores, samples = 0.0, None, []
    for g, trips, p, q in parts:
        v, cores, sample = cpu_baseline(g, trips, p, q, budget_s / len(parts))
        secs += 1.0 / max(v, 1e-12)
        samples.append(f"{g.name}: {sample}")
    return len(parts) / secs, cores, "; ".join(samples)


def run_ours_multi(args):
    """The heterogeneous workload: rows of four grids in one persistent launch."""
    import torch
    from gpusim2grid_b200 import replicas
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=900)
    from gpusim2grid_b200 import RowStatus, compute_many
    from gpusim2grid_b200._native import lib

    parts = _workload(args.workload)
    learned = args.start == "learned"
    prec = lib.PREC_MIXED if args.precision == "mixed" else lib.PREC_FP64
    facades = [_facade(g, trips, p, q, args, local) for g, trips, p, q in parts]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    csrs = [_ids(trips) for _, trips, _, _ in parts]
    sbus = [torch.as_tensor((p + 1j * q) / g.sn_mva, device="cuda") for g, _, p, q in parts]
    n_rows = [p.shape[0] for _, _, p, _ in parts]
    train = []
    learners = []
    if learned:
        for (g, _, _, _), f in zip(parts, facades):
            t0 = time.perf_counter()
            # grids above 2000 buses are costly to solve for training rows: a fifth of the rows
            ls, rep, mix = _train_learned(g, args, local, args.workload,
                                          n_rows=args.train_rows if g.n_bus <= 2000 else args.train_rows // 5)
            learners.append(ls)
            train.append({"grid": g.name, "rows": rep["n_rows"], "unconverged_dropped": rep["n_unconverged"],
                          "t_total_s": round(time.perf_counter() - t0, 2),
                          "val_mse": round(rep["val"][-1], 5) if rep["val"] else None})
            f.set_learned_start(ls, args.refactor_ratio, args.max_reuse)
    for f in facades:
        f.start = "learned" if learned else "flat"
        if args.tune_rates:
            f.autotune(tuple(args.tune_rates), repeats=1)
    ratio, reuse = facades[0]._learned_opts if learned else (0.0, 0)
    strat = {"adaptive": lib.REFACTOR_ADAPTIVE, "base_chord": lib.REFACTOR_BASE_CHORD,
             "refactor_every": lib.REFACTOR_EVERY}[facades[0]._strategy]
    sessions = [f.session for f in facades]
    start_mode = lib.START_ROWS if learned else lib.START_VINIT
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sweeps = []
    chord_log = []  # Newton steps on the shared base factors, per step

    def step():
        pre_ms = 0.0
        if learned:
            bufs = [s.start_rows_buffer(n) for s, n in zip(sessions, n_rows)]
            ev0.record()
            for ls, sb, c, n, b in zip(learners, sbus, csrs, n_rows, bufs):
                ls.start_voltages(sb, c, n, out_ptr=b)
            ev1.record()
            ev1.synchronize()
            pre_ms = ev0.elapsed_time(ev1)
        lib.run_multi(sessions, MAX_ITER, TOL, False, prec, start_mode, 0.0, 0, False, strat, ratio, reuse, learned)
        tm0 = sessions[0].timings()
        ms = sweep_ms = tm0["kernel_ms"]
        chord_log.append(int(tm0["chord_steps"]))
        for f in facades:
            f._ran = True
            ms += f.fp64_fallback()
        sweeps.append(sweep_ms)
        return pre_ms, ms

    for _ in range(args.warmup):
        step()
    clk = ClockSampler(local)
    clk.start()
    replicas.barrier()
    pre, ker = [], []
    torch.cuda.nvtx.range_push("bench_timed")
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a_, b_ = step()
        pre.append(a_)
        ker.append(b_)
    torch.cuda.nvtx.range_pop()
    replicas.barrier()
    clocks = clk.stop()
    total_ms = replicas.max_over_ranks(float(np.sum(pre) + np.sum(ker)), device="cuda")
    fallback_rows = sum(f.fallback_rows for f in facades)
    res = [s.results() for s in sessions]
    n_conv = sum(int((r[2] == RowStatus.CONVERGED).sum()) for r in res)
    iters = np.concatenate([r[3] for r in res])
    n_total = int(sum(n_rows))
    value = world * n_conv * args.steps / (total_ms / 1e3)
    # roofline of the multi-grid sweep launch: each grid's algorithmic bytes
    # per LU and per Newton step times its rows' counts in the last step
    # a step on a grid's shared base factor reads no factor of its own; the
    # chord steps are counted over all grids, so they are split by each
    # grid's share of the Newton steps (an approximation)
    w = 4 if args.precision == "mixed" else 8
    launch_bytes = 0
    chord_steps = chord_log[-1] if chord_log else 0
    steps_all = max(1, int(sum(int(r_[3].sum()) for r_ in res)))
    for s_, (g_, _, _, _), r_ in zip(sessions, parts, res):
        info_ = s_.info()
        b_fact, b_iter = algorithmic_bytes(info_, w)
        b_iter += 16 * g_.n_bus  # each step reads the row's Sbus
        steps_g = int(r_[3].sum())
        shared_g = int(round(chord_steps * steps_g / steps_all))
        launch_bytes += (b_fact * int(s_.factor_counts().sum()) + (b_iter - w * info_["nnz_lu"]) * shared_g
                         + b_iter * (steps_g - shared_g))
    sweep_ms = float(np.mean(sweeps[-args.steps:]))
    achieved_gbs = launch_bytes / (sweep_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()

    def flat_arm(p_, strat_):
        lib.run_multi(sessions, MAX_ITER, TOL, False, p_, lib.START_VINIT, 0.0, 0, False, strat_)
        ms_ = []
        for _ in range(max(1, min(args.steps, 3))):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            lib.run_multi(sessions, MAX_ITER, TOL, False, p_, lib.START_VINIT, 0.0, 0, False, strat_)
            ms_.append(sessions[0].timings()["kernel_ms"])
        r_ = [s.results() for s in sessions]
        return sum(int((x[2] == 0).sum()) for x in r_) / (np.mean(ms_) / 1e3), r_

    fp64_value, res64 = flat_arm(lib.PREC_FP64, lib.REFACTOR_EVERY)
    # the metric counts a row when it converged here and in plain FP64 from
    # flat, to the same solution
    n_counted = sum(_counted(r[0], r[2], r64[0], r64[2]) for r, r64 in zip(res, res64))
    value = world * n_counted * args.steps / (total_ms / 1e3)
    agree, same, mism = 0.0, True, {}
    for (g, _, _, _), r, r64 in zip(parts, res, res64):
        ok = (r[2] == 0) & (r64[2] == 0)
        if ok.any():
            agree = max(agree, float(np.abs(r[0][ok] - r64[0][ok]).max()))
        diff = (r[2] == 0) != (r64[2] == 0)
        mism[g.name] = {"converged_here_only": int(((r[2] == 0) & ~(r64[2] == 0)).sum()),
                        "converged_fp64_only": int((~(r[2] == 0) & (r64[2] == 0)).sum())}
        same = same and not bool(diff.any())
    mixed_flat_value = flat_arm(lib.PREC_MIXED, lib.REFACTOR_ADAPTIVE)[0] if learned else None

    # end to end: host rows in, every grid's voltages / statuses / residuals
    # out (V written by the kernels into each session's page-locked result
    # buffer as rows leave; the rest by one DMA per array)
    for f in facades:
        f.results_to_host = True
    gc.collect()
    gc.freeze()
    e2e_s, e2e_parts = [], []
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            e2e_s, e2e_parts = [], []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f, (g, trips, p, q) in zip(facades, parts):
            _set_rows(f, trips, p, q, g)
        t1 = time.perf_counter()
        kms = compute_many(facades)
        t2 = time.perf_counter()
        outs = [f.results_view()[:3] for f in facades]
        outs = [(v, st, r) for v, r, st in outs]
        t3 = time.perf_counter()
        e2e_s.append(t3 - t0)
        e2e_parts.append((t1 - t0, t2 - t1, t3 - t2, kms / 1e3))
    gc.unfreeze()
    e2e_split = dict(zip(["rows_in_ms", "compute_ms", "results_out_ms", "kernel_ms"],
                         [round(float(x) * 1e3, 2) for x in np.mean(np.array(e2e_parts), axis=0)]))
    n_conv_e2e = sum(_counted(o[0], o[1], r64[0], r64[2]) for o, r64 in zip(outs, res64))
    e2e_value = world * n_conv_e2e / float(np.mean(e2e_s))
    h2d = sum(2 * p.nbytes + 4 * (len(t) + 1) + 4 * sum(len(x) for x in t) for _, t, p, _ in parts)
    d2h = sum(o[0].nbytes + o[1].nbytes + o[2].nbytes for o in outs)

    # base_chord: the multi-grid chord sweep, then the hand-off sweep
    sweep_launches = 2 if strat == lib.REFACTOR_BASE_CHORD else 1
    per_step_launches = sweep_launches + (sum(ls.launches_per_call(n) for ls, n in zip(learners, n_rows))
                                          if learned else 0) + (1 if fallback_rows else 0)
    line = {
        "metric": METRIC,
        "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 mismatch/V, f32 J/LU, bf16 MLP" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": args.workload, "grids": [g.name for g, _, _, _ in parts], "rows": n_total,
                   "rows_per_grid": n_rows, "start": args.start, "precision": args.precision,
                   "strategy": args.strategy, "tol_pu": TOL, "max_iter": MAX_ITER, "launch": "one persistent launch",
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{world}"},
        "rows_converged": n_conv, "rows_counted": n_counted, "rows_fp64_fallback": fallback_rows,
        "mean_iters": round(float(iters.mean()), 3),
        "iters_hist": {int(k): int(v) for k, v in zip(*np.unique(iters, return_counts=True))},
        "ms_split": {"features_mlp_v0": round(float(np.mean(pre)), 4), "sweep_kernel": round(float(np.mean(ker)), 4)},
        "fp64_flat_value": round(fp64_value, 1),
        "speedup_vs_fp64_flat": round(value / world / fp64_value, 3),
        "mixed_flat_value": None if mixed_flat_value is None else round(mixed_flat_value, 1),
        "agreement_with_fp64": {"max_abs_dv_pu": agree, "same_convergence_flags": same, "flag_differences": mism},
        "training": train,
        "plan_tails": [s.info()["tail_dim"] for s in sessions],
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 4), "traffic": None,
                     "note": f"multi-grid chord sweep + hand-off sweep ({round(sweep_ms, 3)} ms per step); peak "
                             f"{peak_kind}; algorithmic bytes = sum over grids of bytes per LU x LUs + bytes per "
                             f"Newton step x steps, a step on the shared base factor without its factor read "
                             f"({chord_steps} of {steps_all} steps) = {launch_bytes}"},
        "e2e": {"value": round(e2e_value, 1), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "split": e2e_split},
        "gpu_launches": args.steps * per_step_launches,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        v, cores, sample = cpu_baseline_multi(parts, args.cpu_budget_s)
        line["cpu_baseline"] = {"value": round(v, 2), "unit": "solves/s", "cores": cores, "kind": "port",
                                "sample": sample, "cpu_model": _cpu_model()}
    replicas.finish()
    if rank == 0:
        print(json.dumps(line))


# ---------------------------------------------------------------- reference arm
def _single_cpu_rate(g, budget_s, threads):
    """Solves/s of the compiled CPU NR (oracle/cpu_nr.cpp) on copies of one
    system, ``threads`` host threads over the copies; about ``budget_s``
    seconds."""
    from oracle import cpu_nr
    Y, V0, S, _, _, pv, pq = g.as_tuple()

    def run(k):
        sb = np.repeat(np.asarray(S, dtype=np.complex128)[None, :], k, axis=0)
        t0 = time.perf_counter()
        _, st, _, _, _ = cpu_nr.sweep(Y, V0, S, pv, pq, sbus_rows=sb, max_iter=MAX_ITER, tol=TOL, threads=threads)
        return int((st == 0).sum()), time.perf_counter() - t0

    conv, dt = run(16 * threads)
    k = max(16 * threads, int(conv / dt * budget_s))
    conv, dt = run(k)
    return conv / dt, k


def run_ours_single(args):
    """The single-solve path: one system (AcPfGPU, the reference's acpf_nr_gpu
    / AcPfGPU facade) solved again from Vinit each step, step-then-test
    iteration as the reference's run_single_system_nr.  value: solves/s from
    the session's device time; e2e: the facade's resolve() with the host
    start voltage in and solve() with the host voltage out, wall time."""
    import torch
    from gpusim2grid_b200 import AcPfGPU, replicas
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=900)
    g, _, _, _ = _workload(args.workload)
    grid = g.as_tuple()
    V0 = grid[1]
    ac = AcPfGPU(grid, precision=args.precision, max_iter=MAX_ITER, tol=TOL, device=local,
                 init_from_n_powerflow=False)
    for _ in range(args.warmup):
        ac.resolve(V0)
    clk = ClockSampler(local)
    clk.start()
    replicas.barrier()
    ks, its = [], []
    for _ in range(args.steps):
        t = ac.resolve(V0)
        ks.append(t.t_kernel_ms)
        its.append(t.nb_iter)
    replicas.barrier()
    clocks = clk.stop()
    total_ms = replicas.max_over_ranks(float(np.sum(ks)), device="cuda")
    value = world * args.steps / (total_ms / 1e3)
    gc.collect()
    e2e_s = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ac.resolve(V0)
        V = ac.solve()
        if i >= args.warmup:
            e2e_s.append(time.perf_counter() - t0)
    e2e_value = world / float(np.mean(e2e_s))
    info = ac.session.info()
    w = 4 if args.precision == "mixed" else 8
    b_fact, b_iter = algorithmic_bytes(info, w)
    it = int(np.mean(its))
    achieved = (b_fact * it + b_iter * it) / (total_ms / args.steps / 1e3) / 1e9
    peak, peak_kind = _peaks()
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64 mismatch/V, f32 J/LU",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": args.workload, "grid": g.name, "rows": 1, "start": "flat", "precision": args.precision,
                   "tol_pu": TOL, "max_iter": MAX_ITER, "schedule": "single solve: step, then test the mismatch "
                   "before it", "parallelism": f"replicas x{world}", "l2": "inputs far below L2 (single solve)"},
        "newton_iters": it,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5), "traffic": None,
                     "note": f"peak {peak_kind}; one 118-bus system is a latency-bound chain of phases on one CTA: "
                             f"algorithmic bytes = {b_fact} per LU + {b_iter} per step, one LU per step"},
        "e2e": {"value": round(e2e_value, 1), "unit": "solves/s", "h2d_bytes_per_step": int(V0.nbytes),
                "d2h_bytes_per_step": int(V.nbytes)},
        "gpu_launches": args.steps,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        v, k = _single_cpu_rate(g, args.cpu_budget_s, 1)
        line["cpu_baseline"] = {"value": round(v, 2), "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": f"{k} solves of the same system on one thread, flat start, compiled FP64 "
                                          f"NR (oracle/cpu_nr.cpp)", "cpu_model": _cpu_model()}
    replicas.finish()
    if rank == 0:
        print(json.dumps(line))


def run_reference(args):
    """The reference's CPU path restated (the reference itself cannot be
    built here): the compiled FP64 Newton-Raphson of oracle/cpu_nr.cpp on
    every host thread, over the same workload's rows.  Each step is one pass
    over all rows, or over an evenly spaced sample sized to about
    --cpu-budget-s seconds when all rows would take longer."""
    rank, world, _ = _dist()
    if rank != 0:
        return
    w = _workload(args.workload)
    if WORKLOADS[args.workload][1] == "single":
        threads = _host_threads()
        g = w[0]
        for _ in range(args.warmup):
            _single_cpu_rate(g, args.cpu_budget_s, threads)
        runs = [_single_cpu_rate(g, args.cpu_budget_s, threads) for _ in range(args.steps)]
        value = float(np.mean([r[0] for r in runs]))
        n = 1
        sample = (f"{runs[-1][1]} solves of the same system, OpenMP over the copies, flat start, compiled FP64 NR "
                  f"(oracle/cpu_nr.cpp)")
        bases = [type("T", (), {"threads": threads})()]
    else:
        multi = isinstance(w, list)
        parts = w if multi else [w]
        bases = [CpuBaseline(g, trips, p, q, args.cpu_budget_s / len(parts)) for g, trips, p, q in parts]

        def one():
            return len(bases) / sum(1.0 / max(b.measure(), 1e-12) for b in bases)

        for _ in range(args.warmup):
            one()
        vals = [one() for _ in range(args.steps)]
        value = float(np.mean(vals))
        n = sum(b.n for b in bases)
        sample = "; ".join(f"{g.name}: {b.sample}" for (g, _, _, _), b in zip(parts, bases))
    print(json.dumps({
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": args.workload, "grid": WORKLOADS[args.workload][0], "rows": n, "start": "flat",
                   "tol_pu": TOL, "max_iter": MAX_ITER},
        "cpu_baseline": {"value": round(value, 2), "unit": "solves/s", "cores": bases[0].threads, "kind": "port",
                         "sample": sample, "cpu_model": _cpu_model()},
        "e2e": {"value": round(value, 2), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (gpusim2grid) needs cuDSS, Eigen and lightsim2grid, none installable here; "
                "this arm times the compiled CPU restatement of its Newton-Raphson (oracle/cpu_nr.cpp, pinned to "
                "oracle/nr_oracle.py, itself pinned to the reference's own Python)",
        "native_so_loaded": _native_maps(),
    }))


if __name__ == "__main__":
    a = _args()
    LOAD_SCALE = float(a.load_scale)
    if a.impl == "reference":
        run_reference(a)
    elif WORKLOADS[a.workload][1] == "single":
        run_ours_single(a)
    elif WORKLOADS[a.workload][1] == "multi":
        run_ours_multi(a)
    else:
        run_ours(a)
