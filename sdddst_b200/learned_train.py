"""Trains the learned correction C of the cluster preconditioner (see
sdddst_b200/learned.py) on the device and writes
sdddst_b200/learned_weights.npz.

    python -m sdddst_b200.learned_train [--jacobians 20000] [--sizes 4096 8192 16384 32768]
                                        [--probes 8] [--lr 1e-5] [--heldout 16] [--settle 10]

Every training step is one call of sdddst_learned_train_step: the device
assembles the Jacobian J(h) of the engine's accepted configuration, builds
its cluster inverse B, draws sign probes Z, runs the network forward, the
loss ||Z - J (B + C) Z||^2 / ||Z||^2 and its gradient with hand-written
kernels (node products and weight gradients on the tensor cores, BF16
operands, FP32 accumulation) and one Adam step on the FP32 master weights
(global-norm clipping at 1, cosine-decayed learning rate).  No PyTorch.

Data: the Jacobians the method itself generates.  Runs of the mixed
learned-preconditioned method (cutoff multiplier 2, precision 1e-5, zero
stress) at N taken in turn from --sizes with seeds other than the benchmark
workload's; after every accepted step the network trains on J(h) and on
J(h/2) of the next step's full and half steps, until --jacobians Jacobians
have been used.  A held-out run (N = 8192, seed 12) provides --heldout
states; the file records their loss with B alone, with the first-order
correction (the starting network: zero output layers) and with the trained
correction.  The file keeps the checkpoint (taken after each run, the start
included) with the lowest held-out loss.  Each step follows the loss relative
to the loss with B alone, so Jacobians of every step size weigh alike, and
each run's first --settle accepted steps (the initial step-size transient)
are skipped.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np


def _engine(n, seed):
    from sdddst_b200 import capi, workloads
    xyb, _ = workloads.dislocations(n, seed)
    return capi.Engine(capi.cli_params(n, 2.0, 1e-5, step_size=1e-6, pairsum=capi.PAIRSUM_FP32,
                                       solver=capi.SOLVER_GMRES_LEARNED), xyb)


def heldout_states(count, w0, settle):
    """(engine, [(configuration, step size), ...]) of a held-out run, from
    its accepted steps after the first `settle`."""
    e = _engine(8192, 12)
    e.learned_train_init(w0)
    states = []
    accepted = 0
    while len(states) < count:
        if e.step():
            accepted += 1
            if accepted > settle:
                sc = e.scalars()
                states.append((e.config(0), sc["step_size"]))
    return e, states


def evaluate(e, states, probes, weights):
    """Mean held-out losses (B alone, B + C) for the given FP32 weights."""
    e.learned_train_init(weights)
    lb = lc = 0.0
    for k, (cfg, h) in enumerate(states):
        sc = e.scalars()
        e.set_state(cfg, h, sc["sim_time"], sc["energy"], sc["strain"], False)
        b, c = e.learned_train_step(h, probes=probes, lr=0.0, seed=10_000 + k, apply=False)
        lb += b
        lc += c
    return lb / len(states), lc / len(states)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jacobians", type=int, default=20000)
    ap.add_argument("--sizes", type=int, nargs="+", default=[4096, 8192, 16384, 32768])
    ap.add_argument("--probes", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-5)
    ap.add_argument("--settle", type=int, default=10,
                    help="accepted steps of each run (and of the held-out run) before its Jacobians are used")
    ap.add_argument("--steps-per-run", type=int, default=400, help="accepted steps before the next run")
    ap.add_argument("--heldout", type=int, default=16)
    ap.add_argument("--out", default=None)
    ap.add_argument("--compare", default=None, help="a weight file whose held-out loss the record also states")
    args = ap.parse_args(argv)
    from sdddst_b200 import build, learned
    build.build()
    log = lambda s: print(s, flush=True)
    t0 = time.time()
    w0 = learned.init_weights(0)
    ev, states = heldout_states(args.heldout, w0, args.settle)
    lb0, lf0 = evaluate(ev, states, args.probes, w0)
    log(f"held-out: B {lb0:.4e}  B + first order {lf0:.4e}")
    lcmp = None
    if args.compare:
        bits = learned.load_weights(args.compare).astype(np.uint32) << 16
        lcmp = evaluate(ev, states, args.probes, bits.view(np.float32))[1]
        log(f"held-out: B + {args.compare} {lcmp:.4e}")
    weights = w0
    best, best_loss, best_at = w0, lf0, 0
    used = 0
    run = 0
    hist = []
    sizes_used = {}
    while used < args.jacobians:
        n = args.sizes[run % len(args.sizes)]
        seed = 100 + run
        e = _engine(n, seed)
        e.learned_train_init(weights)
        # continue the optimiser state across runs: the moments restart, the
        # schedule continues
        accepted = 0
        while accepted < args.steps_per_run + args.settle and used < args.jacobians:
            if not e.step():
                continue
            accepted += 1
            if accepted <= args.settle:  # the initial step-size transient
                continue
            h = e.scalars()["step_size"]
            for hh in (h, 0.5 * h):
                lr = args.lr * 0.5 * (1.0 + math.cos(math.pi * used / args.jacobians))
                b, c = e.learned_train_step(hh, probes=args.probes, lr=lr, seed=used)
                used += 1
                sizes_used[n] = sizes_used.get(n, 0) + 1
                if used % 1000 == 0:
                    log(f"{used} Jacobians ({time.time() - t0:.0f} s): N={n} B {b:.3e}  B + C {c:.3e}")
        weights = e.learned_train_weights()
        e.close()
        hb, hc = evaluate(ev, states, args.probes, weights)
        hist.append({"jacobians": used, "heldout_B": hb, "heldout_learned": hc})
        if hc < best_loss:
            best, best_loss, best_at = weights, hc, used
        log(f"run {run} (N={n}) done: {used} Jacobians, held-out B + C {hc:.4e}")
        run += 1
    # the checkpoint with the lowest held-out loss (the start included)
    bf16 = learned.bf16_bits(best)
    meta = {"trainer": "device (csrc/learned_train.cu)", "jacobians": used, "sizes": sizes_used,
            "probes": args.probes, "lr": args.lr, "settle": args.settle, "runs": run,
            "heldout_states": len(states),
            "heldout_loss": {"B": lb0, "B_plus_first_order": lf0, "B_plus_learned_bf16": best_loss,
                             "B_plus_last": hist[-1]["heldout_learned"] if hist else lf0,
                             "B_plus_compared": lcmp},
            "kept_checkpoint_after_jacobians": best_at, "history": hist, "seconds": time.time() - t0}
    log(json.dumps(meta["heldout_loss"]))
    np.savez(args.out or learned.WEIGHTS_FILE, bf16=bf16, meta=np.array(json.dumps(meta)))


if __name__ == "__main__":
    sys.exit(main())
