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
hot path compiled in place) on a bounded sample of the same workload, see
``reference_arm``.
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
PAIR_F32_DRAM_BYTES_N32768 = 812544 + 8764672  # measured, see the roofline note in main()
PREC = 1e-5
H0 = 1e-6
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
    torch.cuda.synchronize()
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


def cpu_baseline_sample(n_full, sample_n=4096, reps=1):
    """The reference hot path (compiled in place) on a bounded sample: the
    first `sample_n` dislocations of the workload with the same cutoff radius
    (multiplier scaled by sqrt(sample_n / N)); calculateSpeeds and
    calculateJacobian are timed and scaled by the unique-pair ratio
    N(N-1) / (n(n-1)) (both are O(N^2) scans; at fixed radius the Jacobian's
    entries also grow as N^2).  One step attempt of the reference costs 5
    velocity evaluations and 3 assemblies (zero stress,
    simulation.cpp:62-84,435-650); the UMFPACK solve is not counted (it only
    makes the reference slower)."""
    sys.path.insert(0, ROOT)
    from oracle import ref
    from sdddst_b200 import workloads
    if not ref.available("ref"):
        kind = "port"
        if not ref.available("port"):
            subprocess.run(["make", "-s", "port"], cwd=os.path.join(ROOT, "oracle"), check=True)
    else:
        kind = "reference"
    xyb, _ = workloads.dislocations(n_full, SEED)
    xs = np.ascontiguousarray(xyb[:sample_n])
    m_s = CUTOFF_M * np.sqrt(sample_n / n_full)
    sim = ref.Sim(xs, None, ref.params(cutoff_multiplier=m_s, prec=PREC, step_size=H0),
                  "ref" if kind == "reference" else "port")
    t0 = time.perf_counter()
    for _ in range(reps):
        sim.speeds(xs)
    t_sp = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        sim.jacobian(H0, xs)
    t_jac = (time.perf_counter() - t0) / reps
    scale = (n_full * (n_full - 1.0)) / (sample_n * (sample_n - 1.0))
    t_step = (5 * t_sp + 3 * t_jac) * scale
    return {"value": 1.0 / t_step, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": (f"first {sample_n} dislocations of the workload, cutoff radius kept; calculateSpeeds "
                       f"{t_sp:.3f} s + calculateJacobian {t_jac:.3f} s, scaled by N(N-1)/(n(n-1)) = {scale:.1f} "
                       f"to 5 evaluations + 3 assemblies per attempt; solve not counted"),
            "seconds_per_step": t_step}


def reference_arm(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    n = args.n
    steps = max(1, args.steps)
    vals = []
    info = None
    for k in range(args.warmup + steps):
        info = cpu_baseline_sample(n, sample_n=min(n, 2048))
        if k >= args.warmup:
            vals.append(info["seconds_per_step"])
    t = sum(vals) / len(vals)
    v = 1.0 / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"n{n}_m{CUTOFF_M}_seed{SEED}", "N": n, "cutoff_multiplier": CUTOFF_M,
                       "prec": PREC, "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": info["kind"], "sample": info["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_target(args):
    """Small, self-contained launches for ncu captures: the pair-sum kernels
    `reps` times on the workload's configuration, `steps` step attempts, one
    sparse-LU solve (plain FP64 engine, h = 1e-6), or one inference of the
    learned preconditioner correction (h = 1e-7)."""
    from sdddst_b200 import capi
    if args.only == "direct":
        eng, xyb = make_engine(args.n, "fp64", 0, solver=capi.SOLVER_DIRECT)
        rhs = np.random.default_rng(0).standard_normal(args.n)
        x, refinements = eng.solve(1e-6, xyb, rhs)
        print(json.dumps({"target": "direct", "n": args.n, "refinements": refinements, **eng.direct_stats()}))
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


def measure_batch(torch, steps, warmup, pairsum, rank, world, dist=None):
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
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        n = torch.tensor([acc], device="cuda", dtype=torch.float64)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        total_ms, acc = float(t.item()), int(n.item())
    bt.close()
    return {"value": acc / (total_ms * 1e-3) if total_ms > 0 else 0.0, "unit": "accepted system-steps/s",
            "systems": len(sizes), "systems_per_rank": len(mine), "total_dislocations": int(sum(sizes)),
            "steps": steps, "ms_per_step": total_ms / max(1, steps), "tile": info["tile"],
            "pairsum": pairsum, "gpu_launches": launches,
            "config": "N_k ~ U[64, 2048] seed 3, cutoff multiplier 0.5, prec 1e-6, zero stress"}


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
    ap.add_argument("--only", default=None, choices=["pairsum", "step", "direct", "learned"],
                    help="profiling target: launch only the pair-sum kernels (or only steps) and exit")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-realisations measurement")
    ap.add_argument("--no-variants", action="store_true", help="skip the preconditioner variants")
    args = ap.parse_args()
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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    eng, xyb = make_engine(args.n, args.pairsum, local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, accepted, launches = time_steps(torch, eng, args.steps, args.warmup, flush)
    clk = clocks.stop()
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
    # DRAM traffic of one full-size launch (dram__bytes_read.sum + dram__bytes_write.sum, one ncu
    # capture at N=32768, profiles/pair_tiles_f32_n16384.md): positions read, partials mostly in L2
    traffic = PAIR_F32_DRAM_BYTES_N32768 if (args.pairsum == "fp32" and args.n == N_FULL) else None
    roof = {"bound": args.pairsum, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_unit": "bytes per launch", "peak_source": peak_src,
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
            batch = measure_batch(torch, max(2, args.steps // 2), 2, args.pairsum, rank, ws, dist)
        except Exception as ex:  # reported, never required for the main line
            batch = {"error": str(ex)[:200]}

    cpu = None
    if rank == 0 and not args.no_cpu and ws == 1:
        try:
            cpu = cpu_baseline_sample(args.n)
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
                   "solver": "gmres(30) fp64, cluster block-Jacobi preconditioner",
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas" if ws > 1 else "none",
                   "accepted": accepted, "attempts": args.steps, "final_step_size": sc["step_size"],
                   "solver_stats": solver_stats,
                   "gmres_iterations_per_solve": solver_stats["iterations"] / max(1, solver_stats["solves"])},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk,
        "plain_fp64": plain,
        **variants,
        "position_error_vs_fp64": pos_err,
        "precision_16384": precision,
        "batch_512": batch,
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
