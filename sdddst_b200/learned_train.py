"""Trains the learned correction C of the cluster preconditioner (see
sdddst_b200/learned.py) and writes sdddst_b200/learned_weights.npz.

    python -m sdddst_b200.learned_train [--sizes 4096 8192] [--seeds 11 12]
                                        [--attempts 16] [--probes 8] [--iters 2500]

Data: for every accepted configuration of runs of the mixed-precision method
(cutoff multiplier 2, precision 1e-5, zero stress; seeds other than the
benchmark workload's), the Jacobians J(h) and J(h/2) of the next step's
full and half steps, k random sign probes Z and the cluster preconditioner's
B Z (sdddst_precond_apply).  Loss: the probe estimate of the right
preconditioned residual, ||Z - J (B + C) Z||^2 / ||Z||^2.  The last run is
held out for validation; the file records the held-out loss of B alone, of
B plus the analytic first-order correction (c_ij = -1 across blocks) and of
B plus the trained correction.
"""
from __future__ import annotations

import argparse
import json
import random
import sys
import time

import numpy as np


def generate(n, seed, attempts, k, device, log):
    import torch
    from sdddst_b200 import capi, workloads
    from sdddst_b200.learned import Graph
    xyb, _ = workloads.dislocations(n, seed)
    eng = capi.Engine(capi.cli_params(n, 2.0, 1e-5, step_size=1e-6, pairsum=capi.PAIRSUM_FP32), xyb)
    out = []
    for a in range(attempts):
        eng.step()
        sc = eng.scalars()
        h, cut = sc["step_size"], sc["cutoff"]
        cfg = eng.config(0)
        for hh in (h, 0.5 * h):
            rp, col, val, d = eng.jacobian(hh, cfg)
            Z = (torch.randint(0, 2, (k, n), device=device, dtype=torch.float64) * 2 - 1).contiguous()
            BZ = torch.empty_like(Z)
            blk = torch.empty(n, dtype=torch.int32, device=device)
            torch.cuda.synchronize()
            eng.precond_apply(hh, k, Z.data_ptr(), BZ.data_ptr(), blk.data_ptr())
            g = Graph(rp, col, val, d, cfg[:, 0], cfg[:, 1], cut, blk.cpu().numpy(), device)
            Zt, BZt = Z.T.contiguous(), BZ.T.contiguous()
            out.append((g, Zt, Zt - g.apply_J(BZt)))
    log(f"  N={n} seed={seed}: {len(out)} Jacobians, nnz/row {int(rp[-1]) / n:.0f}, final h {h:.3e}")
    eng.close()
    return out


def losses(net, samples):
    import torch
    lb = ln = lt = 0.0
    with torch.no_grad():
        for g, Z, R0 in samples:
            zz = float((Z ** 2).sum())
            lb += float((R0 ** 2).sum()) / zz
            same = g.edge_f[:, 4].double()
            ce = -(1.0 - same)
            R1 = R0 - g.apply_J(g.apply_C(ce, torch.zeros(g.n, device=Z.device, dtype=torch.float64), Z))
            ln += float((R1 ** 2).sum()) / zz
            c_e, c_d = net(g)
            R2 = R0 - g.apply_J(g.apply_C(c_e, c_d, Z))
            lt += float((R2 ** 2).sum()) / zz
    m = max(1, len(samples))
    return lb / m, ln / m, lt / m


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", type=int, nargs="+", default=[4096, 8192])
    ap.add_argument("--seeds", type=int, nargs="+", default=[11, 12])
    ap.add_argument("--attempts", type=int, default=16)
    ap.add_argument("--probes", type=int, default=8)
    ap.add_argument("--iters", type=int, default=2500)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    import torch
    from sdddst_b200 import build, learned
    build.build()
    torch.manual_seed(0)
    random.seed(0)
    dev = "cuda"
    log = lambda s: print(s, flush=True)
    t0 = time.time()
    runs = [(n, s) for n in args.sizes for s in args.seeds]
    data = [generate(n, s, args.attempts, args.probes, dev, log) for n, s in runs]
    train = [x for run in data[:-1] for x in run]
    val = data[-1]
    log(f"data: {len(train)} training, {len(val)} held-out Jacobians in {time.time() - t0:.0f} s")
    net = learned.make_net().to(dev)
    with torch.no_grad():  # start from the correction being zero: M = B
        net.wo.weight.zero_()
        net.wo.bias.zero_()
        net.wd.weight.zero_()
        net.wd.bias.zero_()
    opt = torch.optim.Adam(net.parameters(), lr=args.lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, args.iters)
    hist = []
    for it in range(args.iters):
        g, Z, R0 = random.choice(train)
        c_e, c_d = net(g)
        R = R0 - g.apply_J(g.apply_C(c_e, c_d, Z))
        loss = (R ** 2).sum() / (Z ** 2).sum()
        opt.zero_grad()
        loss.backward()
        torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
        opt.step()
        sched.step()
        if it % 250 == 0 or it == args.iters - 1:
            lb, ln, lt = losses(net, val)
            hist.append({"iter": it, "train": float(loss), "val_B": lb, "val_B_neumann": ln, "val_learned": lt})
            log(f"iter {it}: train {float(loss):.4e}  held-out: B {lb:.4e}  B+neumann {ln:.4e}  learned {lt:.4e}")
    # the weights as the device will use them (BF16), evaluated once more
    bf16 = learned.pack_bf16(net)
    learned.unpack_into(net, bf16)
    lb, ln, lt = losses(net, val)
    meta = {"sizes": args.sizes, "seeds": args.seeds, "attempts": args.attempts, "probes": args.probes,
            "iters": args.iters, "train_jacobians": len(train), "heldout_jacobians": len(val),
            "heldout_loss": {"B": lb, "B_plus_first_order": ln, "B_plus_learned_bf16": lt},
            "history": hist, "seconds": time.time() - t0}
    log(json.dumps(meta["heldout_loss"]))
    np.savez(args.out or learned.WEIGHTS_FILE, bf16=bf16, meta=np.array(json.dumps(meta)))


if __name__ == "__main__":
    sys.exit(main())
