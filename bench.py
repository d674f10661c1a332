"""Benchmark of the implicit-step hot path: accepted steps/s at N=32768.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--pairsum fp32|fp64] [--n N] [--no-plain] [--no-cpu]

Workload: N = 32768 edge dislocations, x, y uniform on [-0.5, 0.5) from seed
4, balanced +-1 Burgers signs, no point defects, zero external stress,
cutoff multiplier 2.0, precision 1e-5 (CLI default), initial step 1e-6.
A "step" is one adaptive implicit step attempt (Simulation::step): a full
step and two half steps, each with a Jacobian solve, the error estimate and
accept/reject; value = accepted steps / device time of the K timed attempts.

The main line is the mixed-precision path (FP32 pair terms with FP64
accumulation, FP64 positions, error ratio and GMRES solve preconditioned by
cluster block-Jacobi); the plain FP64 drop-in (FP64 pair sum, FP64 Jacobian,
device sparse LU in place of UMFPACK) is timed beside it (``plain_fp64``,
with the LU's factorization time and FP64 flop rate under ``lu``) and the
mixed path's position difference after one step from the same state is
reported (``position_error_vs_fp64``).  Inputs are device-resident when the timed
region starts; between timed steps a 256 MiB buffer is written to flush L2.
``learned_precond`` and ``neumann_precond`` time the same mixed path with
the GMRES preconditioner extended by the learned correction C (the
message-passing network of sdddst_b200/learned.py, inferred on the device)
and by its analytic first-order part alone.
``e2e`` repeats the measurement through the C ABI with the state crossing
host<->device every step (pinned host buffers).

With ``--gpus N`` under torchrun every rank steps its own independent
replica (the path does not shard: replicas only); value = total accepted
steps of all ranks / max over ranks of the device time.

``--impl reference`` times the reference's own CPU code (oracle/_ref, the
hot path compiled in place) for one step attempt of the full workload (five
velocity evaluations and three Jacobian assemblies at N = 32768, one core,
UMFPACK solve excluded), see ``reference_arm``; the repo arm's
``cpu_baseline`` times one of each of those calls at full N in a separate
process and composes the same attempt.  The timed window starts after
``--settle`` accepted steps (default 10) and the warm-up; its step-size
range is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "accepted steps/s at N=32768, learned-precond vs plain GPU, ≤1e-8 pos error"
UNIT = "steps/s"
N_FULL = 32768
SEED = 4
CUTOFF_M = 2.0
# DRAM bytes (read + write) of one FP32 pair-sum launch at N = 32768, recorded
# from one ncu capture of that kernel (0.81 MB read, 8.76 MB written); not
# measured by this script, which has no access to the DRAM counters.
PAIR_F32_DRAM_BYTES_N32768_RECORDED = 812544 + 8764672
PREC = 1e-5
H0 = 1e-6
# GMRES(30) stops at this relative residual on the learned-preconditioner
# workload (its stated tolerance); the plain path's sparse LU refines to 1e-13.
GMRES_TOL = 1e-10
# Pair-sum FLOP convention: tau_xy = 130 FP operations per unique pair.
FLOP_PER_PAIR = 130.0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _vector_peaks(device):
    """FP64 / FP32 FMA peaks of this GPU, measured now by the library's
    calibration kernel (sdddst_vector_peaks)."""
    from sdddst_b200 import capi
    try:
        f64, f32 = capi.vector_peaks(device)
        return {"fp64_tflops": f64, "fp32_tflops": f32}
    except Exception:
        return {}


def make_engine(n, pairsum, device, solver=None):
    from sdddst_b200 import capi, workloads
    xyb, _ = workloads.dislocations(n, SEED)
    extra = {} if solver is None else {"solver": solver}
    if solver is None or solver not in (capi.SOLVER_DIRECT, capi.SOLVER_DIRECT_MIXED):
        extra["solver_tol"] = GMRES_TOL
    prm = capi.cli_params(n, CUTOFF_M, PREC, step_size=H0, device=device,
                          pairsum=capi.PAIRSUM_FP32 if pairsum == "fp32" else capi.PAIRSUM_FP64, **extra)
    return capi.Engine(prm, xyb), xyb


def time_steps(torch, eng, steps, warmup, flush, per_kernel=True):
    """Device time of `steps` step attempts after `warmup` untimed ones."""
    stream = torch.cuda.ExternalStream(eng.stream())
    for _ in range(warmup):
        eng.step()
    torch.cuda.synchronize()
    total_ms = 0.0
    accepted = 0
    l0 = eng.launches()
    s0 = eng.solver_stats()
    hs = [eng.scalars()["step_size"]]
    for _ in range(steps):
        flush.zero_()  # L2 flush between timed steps (outside the events)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        accepted += eng.step()
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
        hs.append(eng.scalars()["step_size"])
    torch.cuda.synchronize()
    time_steps.last_h = (min(hs), max(hs))
    s1 = eng.solver_stats()
    time_steps.last_solver = {"solves": s1[0] - s0[0], "iterations": s1[1] - s0[1]}
    return total_ms, accepted, eng.launches() - l0


def time_e2e(torch, eng, steps, flush):
    """Same metric through the C ABI with host buffers: every step uploads
    the configuration from pinned host memory and downloads the result."""
    n = eng.n
    host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    eng.download_positions(host.data_ptr())
    stream = torch.cuda.ExternalStream(eng.stream())
    total_ms, accepted = 0.0, 0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.upload_positions(host.data_ptr(), False)
        accepted += eng.step()
        eng.download_positions(host.data_ptr())
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
    return total_ms, accepted, 8 * n, 8 * n


def pair_kernel_time(eng, reps=3):
    """Mean device time of one pair-sum launch on the accepted configuration,
    timed by the library with CUDA events on the engine's stream."""
    return eng.profile_pair_sum(reps)


def position_error(eng_mixed, eng_plain):
    """One step from the same accepted state on both paths; max |dx|."""
    x = eng_plain.config(0)
    sc = eng_plain.scalars()
    for e in (eng_mixed, eng_plain):
        e.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
    am, ap = eng_mixed.step(), eng_plain.step()
    errs = [float(np.abs(eng_mixed.config(w)[:, 0] - eng_plain.config(w)[:, 0]).max()) for w in (1, 2, 3)]
    return max(errs), am == ap


def measure_precision(torch, steps, flush, device):
    """The precision workload: N=16384 (seed 2), cutoff multiplier 1, FP32
    pair terms with compensated FP64 accumulation, FP32 Jacobian values, FP32
    sparse LU refined in FP64 to a 1e-12 relative residual, against the plain
    FP64 path (FP64 pair sum, FP64 LU); velocity error on the initial
    configuration and position error one accepted step from the same state."""
    from sdddst_b200 import capi, workloads
    n = 16384
    xyb, _ = workloads.dislocations(n, 2)
    mk = lambda ps, sv: capi.Engine(capi.cli_params(n, 1.0, PREC, step_size=H0, device=device, pairsum=ps,
                                                    solver=sv, solver_tol=1e-12), xyb)
    e32 = mk(capi.PAIRSUM_FP32, capi.SOLVER_DIRECT_MIXED)
    e64 = mk(capi.PAIRSUM_FP64, capi.SOLVER_DIRECT)
    v32, _ = e32.speeds(xyb)
    v64, _ = e64.speeds(xyb)
    out = {"config": "N=16384 seed 2, cutoff multiplier 1, prec 1e-5, solves refined to 1e-12",
           "velocity_error_rel": float(np.abs(v32 - v64).max() / np.abs(v64).max())}
    for name, e in (("fp32_lu_refined", e32), ("fp64_lu", e64)):
        ms, acc, _ = time_steps(torch, e, steps, 3, flush)
        out[name] = {"value": acc / (ms * 1e-3) if ms > 0 else 0.0, "unit": UNIT, "ms_per_step": ms / steps,
                     "accepted": acc}
    err = None
    for _ in range(10):
        x, sc = e64.config(0), e64.scalars()
        for e in (e32, e64):
            e.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
        a32, a64 = e32.step(), e64.step()
        if a64 and a32:
            err = max(float(np.abs(e32.config(w)[:, 0] - e64.config(w)[:, 0]).max()) for w in (1, 2, 3))
            break
    out["position_error_one_step"] = err
    e32.close()
    e64.close()
    return out


def _ref_sim(n_full):
    """The reference hot path compiled in place (oracle/_ref) on the full
    workload, or the oracle port where the reference could not be built."""
    from oracle import ref
    from sdddst_b200 import workloads
    kind = "reference" if ref.available("ref") else "port"
    if kind == "port" and not ref.available("port"):
        subprocess.run(["make", "-s", "port"], cwd=os.path.join(ROOT, "oracle"), check=True)
    xyb, _ = workloads.dislocations(n_full, SEED)
    sim = ref.Sim(xyb, None, ref.params(cutoff_multiplier=CUTOFF_M, prec=PREC, step_size=H0),
                  "ref" if kind == "reference" else "port")
    return sim, xyb, kind


def _jacobian_cap(n_full):
    """Entry capacity of the reference Jacobian export at the workload's
    cutoff (one call, no retry): N (1 + 1.3 pi r^2 N) with r the pattern
    radius (1 + sqrt(36.8)) c."""
    c = CUTOFF_M / np.sqrt(n_full)
    r = c * (1.0 + np.sqrt(36.8))
    return int(n_full * (1.0 + 1.3 * min(1.0, np.pi * r * r) * n_full)) + n_full + 1024


def cpu_full_calls(n_full, speeds=1, jacobians=1):
    """Times the reference's own calculateSpeeds (simulation.cpp:86-131) and
    calculateJacobian (simulation.cpp:236-384) on the FULL workload
    configuration, one core (the reference is single-threaded); returns the
    per-call seconds of each kind."""
    sim, xyb, kind = _ref_sim(n_full)
    t_sp, t_jac = [], []
    for _ in range(speeds):
        t0 = time.perf_counter()
        sim.speeds(xyb)
        t_sp.append(time.perf_counter() - t0)
    cap = _jacobian_cap(n_full)
    for _ in range(jacobians):
        t0 = time.perf_counter()
        sim.jacobian(H0, xyb, cap=cap)
        t_jac.append(time.perf_counter() - t0)
    return {"kind": kind, "t_speeds": t_sp, "t_jacobian": t_jac}


def cpu_baseline_worker(args):
    """Subprocess body of the repo arm's CPU baseline: one full-N call of
    the kind --cpu-baseline-worker names, on one core."""
    which = args.cpu_baseline_worker
    print(json.dumps(cpu_full_calls(args.n, int(which == "speeds"), int(which == "jacobian"))), flush=True)


def start_cpu_baseline(n):
    """Starts the CPU baseline: one full-N calculateSpeeds and one full-N
    calculateJacobian, each in its own process on its own host core, beside
    the GPU measurements (about 75 s each at N = 32768)."""
    return [subprocess.Popen([sys.executable, os.path.abspath(__file__), "--cpu-baseline-worker", which,
                              "--n", str(n)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
            for which in ("speeds", "jacobian")]


def finish_cpu_baseline(procs, timeout=900):
    res = []
    for proc in procs:
        out, err = proc.communicate(timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(err.strip().splitlines()[-1] if err.strip() else f"rc {proc.returncode}")
        res.append(json.loads(out.strip().splitlines()[-1]))
    r = {"kind": res[0]["kind"], "t_speeds": res[0]["t_speeds"], "t_jacobian": res[1]["t_jacobian"]}
    t_sp, t_jac = r["t_speeds"][0], r["t_jacobian"][0]
    t_step = 5 * t_sp + 3 * t_jac
    return {"value": 1.0 / t_step, "unit": UNIT, "cores": 1, "kind": r["kind"],
            "sample": (f"full N={N_FULL} workload configuration: one calculateSpeeds {t_sp:.2f} s and one "
                       f"calculateJacobian {t_jac:.2f} s of the reference on one core, composed as an attempt's "
                       f"5 velocity evaluations + 3 assemblies (zero stress, simulation.cpp:62-84,435-650); "
                       f"UMFPACK solve excluded"),
            "seconds_per_step": t_step}


def reference_arm(args):
    """The reference's own CPU code for one step attempt at the full workload:
    the five calculateSpeeds and three calculateJacobian calls of a
    zero-stress attempt (simulation.cpp:62-84,435-650) at N = 32768.  The
    reference is single-threaded and an attempt runs its calls one after
    the other on one core, so the attempt's time is the sum of the eight
    calls' times; to keep the run within a few minutes the eight calls run
    at once, each in its own process on its own host core (the calls are
    compute-bound; they share no data), and their times are summed.  The
    UMFPACK factorization and solve are excluded (UMFPACK is not installed;
    the harness's stand-in LU would only make the reference slower).  One
    attempt is timed whatever --steps asks for."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    n = args.n
    kinds = ["speeds", "jacobian", "speeds", "speeds", "jacobian", "speeds", "jacobian", "speeds"]
    t0 = time.perf_counter()
    procs = [subprocess.Popen([sys.executable, os.path.abspath(__file__), "--cpu-baseline-worker", which,
                               "--n", str(n)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for which in kinds]
    calls, kind = [], None
    for which, proc in zip(kinds, procs):
        out, err = proc.communicate(timeout=1800)
        if proc.returncode != 0:
            raise RuntimeError(err.strip().splitlines()[-1] if err.strip() else f"rc {proc.returncode}")
        r = json.loads(out.strip().splitlines()[-1])
        kind = r["kind"]
        calls.append((which, (r["t_speeds"] if which == "speeds" else r["t_jacobian"])[0]))
    wall = time.perf_counter() - t0
    t = sum(c for _, c in calls)
    v = 1.0 / t
    t_sp = [c for w, c in calls if w == "speeds"]
    t_jac = [c for w, c in calls if w == "jacobian"]
    sample = (f"one zero-stress step attempt of the reference at the full N={n} configuration: 5 calculateSpeeds "
              f"({min(t_sp):.1f}-{max(t_sp):.1f} s each) and 3 calculateJacobian ({min(t_jac):.1f}-{max(t_jac):.1f} s "
              f"each), each call on its own core at the same time ({wall:.0f} s wall), summed to the {t:.1f} s "
              f"one core takes for the attempt; UMFPACK solve excluded")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": 1,
            "requested_steps": args.steps, "warmup": 0, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"n{n}_m{CUTOFF_M}_seed{SEED}", "N": n, "cutoff_multiplier": CUTOFF_M,
                       "prec": PREC, "parallelism": "none (single-threaded reference; calls timed concurrently)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_target(args):
    """Small, self-contained launches for ncu captures: the pair-sum kernels
    `reps` times on the workload's configuration, `steps` step attempts, one
    sparse-LU solve (plain FP64 engine, h = 1e-6), one inference of the
    learned preconditioner correction (h = 1e-7), or the eigenvalue analysis
    of one configuration (`--n` dislocations, 64 point defects; `reps` timed
    calls after a first one)."""
    from sdddst_b200 import capi
    if args.only in ("direct", "direct_mixed"):
        mixed = args.only == "direct_mixed"
        eng, xyb = make_engine(args.n, "fp32" if mixed else "fp64", 0,
                               solver=capi.SOLVER_DIRECT_MIXED if mixed else capi.SOLVER_DIRECT)
        rhs = np.random.default_rng(0).standard_normal(args.n)
        x, refinements = eng.solve(1e-6, xyb, rhs)
        print(json.dumps({"target": args.only, "n": args.n, "refinements": refinements, **eng.direct_stats()}))
        eng.close()
        return
    if args.only == "ev":
        import torch
        print(json.dumps({"target": "ev", **measure_ev(torch, 0, cpu=False, n=args.n, reps=args.reps)}))
        return
    if args.only == "learned_train":
        # device training steps of the learned correction on J(h) of the
        # workload's configuration at a step size of its settled window
        # (h = 1e-9): `reps` timed steps (each waits for its losses) after one
        from sdddst_b200 import learned
        eng, _ = make_engine(args.n, args.pairsum, 0, solver=capi.SOLVER_GMRES_LEARNED)
        eng.learned_train_init(learned.init_weights(0))
        lb, lc = eng.learned_train_step(1e-9, probes=8, lr=1e-5, seed=0)
        t0 = time.perf_counter()
        for r in range(args.reps):
            eng.learned_train_step(1e-9, probes=8, lr=1e-5, seed=1 + r)
        dt = (time.perf_counter() - t0) / max(1, args.reps)
        print(json.dumps({"target": "learned_train", "n": args.n, "ms_per_step": dt * 1e3, "h": 1e-9,
                          "loss_B": lb, "loss_B_plus_first_order": lc}))
        eng.close()
        return
    if args.only == "learned":
        eng, _ = make_engine(args.n, args.pairsum, 0, solver=capi.SOLVER_GMRES_LEARNED)
        eng.set_preconditioner_weights()
        c = eng.learned_correction(1e-7)
        print(json.dumps({"target": "learned", "n": args.n, "nnz": int(c.size)}))
        eng.close()
        return
    eng, _ = make_engine(args.n, args.pairsum, 0)
    if args.only == "pairsum":
        ms = eng.profile_pair_sum(args.reps)
        print(json.dumps({"target": "pairsum", "n": args.n, "pairsum": args.pairsum, "ms_per_launch": ms}))
    else:
        # `warmup` untimed attempts (the step size adapts), then `steps`
        # attempts inside the NVTX range "steps" (ncu --nvtx --nvtx-include steps/)
        import torch
        for _ in range(args.warmup):
            eng.step()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("steps")
        acc = sum(eng.step() for _ in range(args.steps))
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"target": "step", "n": args.n, "accepted": acc, "steps": args.steps,
                          "warmup": args.warmup}))
    eng.close()


def _ref_attempt_seconds(args):
    """One zero-stress step attempt of the reference (5 calculateSpeeds + 3
    calculateJacobian, simulation.cpp:62-84,435-650) on one system, one core."""
    n, seed, m = args
    sys.path.insert(0, ROOT)
    from oracle import ref
    from sdddst_b200 import workloads
    xyb, _ = workloads.dislocations(int(n), int(seed))
    kind = "ref" if ref.available("ref") else "port"
    sim = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=1e-6, step_size=H0), kind)
    t0 = time.perf_counter()
    for what in ("s", "j", "s", "s", "j", "s", "j", "s"):
        if what == "s":
            sim.speeds(xyb)
        else:
            sim.jacobian(H0, xyb, cap=max(1024, int(n) * 256))
    return time.perf_counter() - t0, kind


def cpu_batch_baseline(sizes, seeds, accept_fraction, procs=8, sample=8):
    """The reference on `procs` host cores for the batched workload: the
    realisations are independent, so P single-threaded reference processes
    step P systems at once.  Sample: `sample` systems of the workload at
    evenly spaced size quantiles, one attempt each (one per process, all at
    once); the attempt time t(N) = a N^2 is fitted to them, summed over all
    systems and divided by P (perfect packing), and the attempts/s converted
    to accepted system-steps/s with the GPU run's acceptance fraction."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    order = np.argsort(sizes)
    pick = order[np.linspace(0, len(sizes) - 1, sample).round().astype(int)]
    jobs = [(int(sizes[k]), int(seeds[k]), 0.5) for k in pick]
    with ProcessPoolExecutor(max_workers=min(procs, sample), mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_ref_attempt_seconds, jobs))
    ts = np.array([r[0] for r in res])
    ns = np.array([j[0] for j in jobs], dtype=np.float64)
    a = float(np.sum(ts * ns ** 2) / np.sum(ns ** 4))
    total = a * float(np.sum(np.asarray(sizes, dtype=np.float64) ** 2))
    wall = total / procs
    attempts_per_s = len(sizes) / wall
    return {"value": attempts_per_s * accept_fraction, "unit": "accepted system-steps/s", "cores": procs,
            "kind": "reference" if res[0][1] == "ref" else "port",
            "sample": (f"{sample} systems of the workload at size quantiles (N = {int(ns.min())}..{int(ns.max())}), "
                       f"one reference attempt each (5 calculateSpeeds + 3 calculateJacobian, one core per system, "
                       f"{sample} at once, {ts.max():.1f} s), t(N) = {a:.3e} N^2 s summed over the "
                       f"{len(sizes)} systems on {procs} cores, times the GPU run's acceptance "
                       f"{accept_fraction:.3f}; solve excluded")}


def measure_batch(torch, steps, warmup, pairsum, rank, world, dist=None, cpu=False):
    """The batched workload: 512 independent realisations, N_k uniform in
    [64, 2048] (seed 3), cutoff multiplier 0.5, zero stress, all stepped
    together; ranks step their LPT share.  Value: accepted system-steps/s of
    the whole job (sum over systems and ranks / max device time)."""
    from sdddst_b200 import capi, sharding, workloads
    sizes = workloads.batch_sizes(workloads.BATCH_COUNT, workloads.BATCH_SEED)
    mine = sharding.rank_share(sizes, rank, world)
    systems = [workloads.dislocations(int(sizes[k]), workloads.BATCH_SEED * 100003 + k)[0] for k in mine]
    prm = capi.default_params(cutoff_multiplier=workloads.BATCH_M, prec=1e-6, step_size=H0,
                              pairsum=capi.PAIRSUM_FP32 if pairsum == "fp32" else capi.PAIRSUM_FP64)
    bt = capi.Batch(prm, systems)
    info = bt.info()
    stream = torch.cuda.ExternalStream(info["stream"])
    for _ in range(warmup):
        bt.step()
    torch.cuda.synchronize()
    total_ms, acc = 0.0, 0
    l0 = bt.info()["launches"]
    for _ in range(steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        acc += int(bt.step().sum())
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
    launches = bt.info()["launches"] - l0
    stats = bt.stats()
    attempts = len(mine) * steps
    # roofline of its dominant kernel: the pair sum over all systems' tiles
    pair_ms, pairs = bt.profile_pair_sum(3)
    vp = _vector_peaks(torch.cuda.current_device())
    peak = vp.get("fp32_tflops" if pairsum == "fp32" else "fp64_tflops")
    ach = FLOP_PER_PAIR * pairs / (pair_ms * 1e-3) / 1e12 if pair_ms > 0 else 0.0
    roof = {"bound": pairsum, "achieved": ach, "peak": peak, "unit": "TFLOP/s",
            "frac": ach / peak if peak else None, "kernel": "batch_pair_kernel (all systems, one launch)",
            "work": f"{FLOP_PER_PAIR:.0f} FLOP x sum_k N_k(N_k-1)/2 = {pairs:.3e} pairs", "ms": pair_ms,
            "peak_source": "measured (FMA chain microbenchmark, sdddst_vector_peaks)", "traffic": None}
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        n = torch.tensor([acc], device="cuda", dtype=torch.float64)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        total_ms, acc = float(t.item()), int(n.item())
    bt.close()
    out = {"value": acc / (total_ms * 1e-3) if total_ms > 0 else 0.0, "unit": "accepted system-steps/s",
           "systems": len(sizes), "systems_per_rank": len(mine), "total_dislocations": int(sum(sizes)),
           "steps": steps, "ms_per_step": total_ms / max(1, steps), "tile": info["tile"],
           "pairsum": pairsum, "gpu_launches": launches, "graph_replay": bool(stats["graph"]),
           "redone_steps": stats["redone"], "roofline": roof,
           "config": "N_k ~ U[64, 2048] seed 3, cutoff multiplier 0.5, prec 1e-6, zero stress"}
    if cpu and rank == 0:
        try:
            seeds = [workloads.BATCH_SEED * 100003 + k for k in range(len(sizes))]
            out["cpu_baseline"] = cpu_batch_baseline(sizes, seeds, acc / max(1, attempts))
        except Exception as ex:
            out["cpu_baseline"] = {"value": None, "kind": "unavailable", "sample": str(ex)[:200]}
    return out


def measure_ev(torch, local, cpu=True, n=4096, p=64, reps=3):
    """The eigenvalue analysis (--ev-analyzation) of one configuration:
    N = 4096 dislocations (seed 4) with 64 point defects, fixed-rate stress
    1e-3 at t = 1: Hessian, eigenpairs (cuSOLVER dsyevd), observables and
    the eigenvalue derivatives, the first 10 eigenvectors read back.  Device
    phase times from CUDA events; `value` = analysed configurations per
    second end to end through the C ABI (host configuration in, host
    results out).  CPU baseline: the oracle's Hessian (C, one core) and
    numpy.linalg.eigh (LAPACK syevd, all host threads) on an N = 2048 sample
    of the same workload, scaled by N^2 and N^3."""
    import time
    from sdddst_b200 import capi, workloads
    xyb, pd = workloads.dislocations(n, SEED, p)
    prm = capi.cli_params(n, 1.0, 1e-6, p=p, pd_scaling=True, stress_kind=capi.STRESS_FIXED_RATE, stress_rate=1e-3,
                          device=local)
    e = capi.Engine(prm, xyb, pd)
    e.ev_analyze(xyb, sim_time=1.0, nvec=10, deriv=True)  # handles, workspaces
    torch.cuda.synchronize()
    walls, phases = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        e.ev_analyze(xyb, sim_time=1.0, nvec=10, deriv=True)
        walls.append(time.perf_counter() - t0)
        phases.append(e.ev_timings())
    e.close()
    best = min(range(reps), key=lambda k: walls[k])
    ph = phases[best]
    pairs = n * (n - 1) / 2.0
    out = {"value": 1.0 / walls[best], "unit": "configurations/s", "n": n, "point_defects": p,
           "config": "seed 4, fixed-rate stress 1e-3 at t = 1, 10 eigenvectors, derivatives on",
           "ms": {k: v for k, v in ph.items()}, "wall_ms": walls[best] * 1e3,
           "hessian_pairs_per_s": pairs / (ph["hessian"] * 1e-3) if ph["hessian"] > 0 else None,
           "eigensolver": "cuSOLVER Xsyevd (divide and conquer), FP64"}
    if cpu:
        import os
        from oracle import ref
        m = 2048
        xs, pds = workloads.dislocations(m, SEED, p)
        t0 = time.perf_counter()
        H = ref.ev_hessian(xs, pds)
        t_h = time.perf_counter() - t0
        t0 = time.perf_counter()
        np.linalg.eigh(H)
        t_e = time.perf_counter() - t0
        per = t_h * (n / m) ** 2 + t_e * (n / m) ** 3
        out["cpu_baseline"] = {"value": 1.0 / per, "unit": "configurations/s", "cores": os.cpu_count(),
                               "kind": "port",
                               "sample": f"N={m} of the workload: oracle Hessian {t_h:.2f} s (C, one core) + "
                                         f"numpy.linalg.eigh {t_e:.2f} s (LAPACK syevd, all threads), scaled by "
                                         f"N^2 and N^3 to N={n}; observables and derivatives excluded"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairsum", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--n", type=int, default=N_FULL)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only", default=None,
                    choices=["pairsum", "step", "direct", "direct_mixed", "learned", "learned_train", "ev"],
                    help="profiling target: launch only the pair-sum kernels (or only steps) and exit")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-realisations measurement")
    ap.add_argument("--no-variants", action="store_true", help="skip the preconditioner variants")
    ap.add_argument("--no-ev", action="store_true", help="skip the eigenvalue-analysis measurement")
    ap.add_argument("--settle", type=int, default=10,
                    help="accepted steps run before the warm-up (the metric's window starts at step 10)")
    ap.add_argument("--cpu-baseline-worker", default=None, choices=["speeds", "jacobian"], help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cpu_baseline_worker:
        cpu_baseline_worker(args)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.only:
        profile_target(args)
        return

    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from sdddst_b200 import build
    build.build()
    cpu_proc = None
    if rank == 0 and not args.no_cpu and ws == 1:
        cpu_proc = start_cpu_baseline(args.n)  # on its own host core, beside the GPU measurements
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    eng, xyb = make_engine(args.n, args.pairsum, local)
    # the metric's window starts after the initial step-size transient:
    # `settle` accepted steps (untimed, before the warm-up)
    settled = 0
    for _ in range(20 * max(1, args.settle)):
        if settled >= args.settle:
            break
        settled += eng.step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, accepted, launches = time_steps(torch, eng, args.steps, args.warmup, flush)
    clk = clocks.stop()
    h_window = list(time_steps.last_h)
    solver_stats = dict(time_steps.last_solver)
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        acc = torch.tensor([accepted], device="cuda", dtype=torch.float64)
        dist.all_reduce(acc, op=dist.ReduceOp.SUM)
        total_ms, accepted_all = float(t.item()), float(acc.item())
    else:
        accepted_all = accepted
    value = accepted_all / (total_ms * 1e-3) if total_ms > 0 else 0.0

    # e2e through the C ABI with host buffers
    e2e_ms, e2e_acc, h2d, d2h = time_e2e(torch, eng, args.steps, flush)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        acc = torch.tensor([e2e_acc], device="cuda", dtype=torch.float64)
        dist.all_reduce(acc, op=dist.ReduceOp.SUM)
        e2e_ms, e2e_acc = float(t.item()), float(acc.item())
    e2e_value = e2e_acc / (e2e_ms * 1e-3) if e2e_ms > 0 else 0.0

    # roofline of the dominant kernel: the pair sum
    t_pair_ms = pair_kernel_time(eng)
    pairs = args.n * (args.n - 1) / 2.0
    achieved = FLOP_PER_PAIR * pairs / (t_pair_ms * 1e-3) / 1e12
    vp = _vector_peaks(local)
    key = "fp32_tflops" if args.pairsum == "fp32" else "fp64_tflops"
    peak = vp.get(key)
    peak_src = "measured (FMA chain microbenchmark, sdddst_vector_peaks)" if peak else "nominal"
    if not peak:
        peak = 80.0 if args.pairsum == "fp32" else 40.0
    # DRAM traffic of one full-size launch (dram__bytes_read.sum + dram__bytes_write.sum of one ncu
    # capture, recorded above): positions read, partials mostly in L2
    traffic = PAIR_F32_DRAM_BYTES_N32768_RECORDED if (args.pairsum == "fp32" and args.n == N_FULL) else None
    roof = {"bound": args.pairsum, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_unit": "bytes per launch",
            "traffic_source": "recorded from one ncu capture of this kernel at this size (not measured in this run)",
            "peak_source": peak_src,
            "kernel": "pair_tiles_kernel (one velocity evaluation)",
            "work": f"{FLOP_PER_PAIR:.0f} FLOP x N(N-1)/2 unique pairs", "ms": t_pair_ms}

    plain = None
    pos_err = None
    if not args.no_plain:
        # the plain drop-in: FP64 pair sum, FP64 Jacobian, device sparse LU
        from sdddst_b200 import capi
        eng_p, _ = make_engine(args.n, "fp64", local, solver=capi.SOLVER_DIRECT)
        p_steps = max(3, args.steps // 2)
        p_ms, p_acc, p_launch = time_steps(torch, eng_p, p_steps, 3, flush)
        plain = {"value": p_acc / (p_ms * 1e-3) if p_ms > 0 else 0.0, "unit": UNIT,
                 "ms_per_step": p_ms / p_steps, "steps": p_steps, "accepted": p_acc, "gpu_launches": p_launch,
                 "pairsum": "fp64", "solver": "sparse LU fp64 (multifrontal, nested dissection), refined to 1e-13"}
        try:
            h_now = eng_p.scalars()["step_size"]
            f_ms, s_ms = eng_p.profile_direct(h_now, 2)
            st = eng_p.direct_stats()
            f64 = vp.get("fp64_tflops") or 40.0
            ach = st["lu_flops"] / (f_ms * 1e-3) / 1e12 if f_ms > 0 else 0.0
            plain["lu"] = {"bound": "fp64", "flops_per_factorization": st["lu_flops"], "factor_ms": f_ms,
                           "solve_ms": s_ms, "achieved": ach, "peak": f64, "unit": "TFLOP/s", "frac": ach / f64,
                           "fronts": st["fronts"], "tree_depth": st["depth"],
                           "front_gb": st["front_doubles"] * 8 / 1e9, "perturbed_pivots": st["perturbed_pivots"]}
        except Exception as ex:
            plain["lu"] = {"error": str(ex)[:200]}
        if args.pairsum == "fp32":
            err, same = position_error(eng, eng_p)
            pos_err = {"max_abs": err, "same_decision": same}
        eng_p.close()

    # the preconditioner variants of the same mixed path: cluster blocks plus
    # the learned correction, and plus its analytic first-order part alone
    variants = {}
    if not args.no_variants:
        from sdddst_b200 import capi
        for name, solver in (("learned_precond", capi.SOLVER_GMRES_LEARNED),
                             ("neumann_precond", capi.SOLVER_GMRES_NEUMANN)):
            try:
                ev, _ = make_engine(args.n, args.pairsum, local, solver=solver)
                if solver == capi.SOLVER_GMRES_LEARNED:
                    ev.set_preconditioner_weights()
                v_steps = max(3, args.steps // 2)
                v_ms, v_acc, v_launch = time_steps(torch, ev, v_steps, 3, flush)
                st = time_steps.last_solver
                variants[name] = {"value": v_acc / (v_ms * 1e-3) if v_ms > 0 else 0.0, "unit": UNIT,
                                  "ms_per_step": v_ms / v_steps, "steps": v_steps, "accepted": v_acc,
                                  "gpu_launches": v_launch,
                                  "gmres_iterations_per_solve": st["iterations"] / max(1, st["solves"])}
                ev.close()
            except Exception as ex:
                variants[name] = {"error": str(ex)[:200]}

    precision = None
    if not args.no_variants:
        try:
            precision = measure_precision(torch, max(3, args.steps // 2), flush, local)
        except Exception as ex:
            precision = {"error": str(ex)[:200]}

    batch = None
    if not args.no_batch:
        try:
            batch = measure_batch(torch, max(2, args.steps // 2), 2, args.pairsum, rank, ws, dist,
                                  cpu=not args.no_cpu and ws == 1)
        except Exception as ex:  # reported, never required for the main line
            batch = {"error": str(ex)[:200]}

    ev_line = None
    if not args.no_ev and rank == 0:
        try:
            ev_line = measure_ev(torch, local, cpu=not args.no_cpu and ws == 1)
        except Exception as ex:
            ev_line = {"error": str(ex)[:200]}

    cpu = None
    if cpu_proc is not None:
        try:
            cpu = finish_cpu_baseline(cpu_proc)
            cpu.pop("seconds_per_step", None)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "unavailable", "sample": str(ex)[:200]}

    sc = eng.scalars()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.pairsum == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": f"n{args.n}_m{CUTOFF_M}_seed{SEED}", "N": args.n, "cutoff_multiplier": CUTOFF_M,
                   "prec": PREC, "initial_step": H0, "pairsum": args.pairsum,
                   "solver": "gmres(30) fp64 to a 1e-10 relative residual, cluster block-Jacobi preconditioner",
                   "arms": "value: the fastest preconditioner (cluster); learned_precond: the learned correction; "
                           "plain_fp64: the plain FP64 direct-solve path",
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas" if ws > 1 else "none",
                   "accepted": accepted, "attempts": args.steps, "final_step_size": sc["step_size"],
                   "window": f"attempts after {settled} accepted steps and {args.warmup} warm-up attempts",
                   "step_size_range": h_window,
                   "solver_stats": solver_stats,
                   "gmres_iterations_per_solve": solver_stats["iterations"] / max(1, solver_stats["solves"])},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "accepted": e2e_acc, "attempts": args.steps, "ms_per_step": e2e_ms / max(1, args.steps)},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk,
        "plain_fp64": plain,
        **variants,
        "position_error_vs_fp64": pos_err,
        "precision_16384": precision,
        "batch_512": batch,
        "ev_analysis_4096": ev_line,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
