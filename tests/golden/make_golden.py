"""Generates the golden fixtures in this folder from the reference hot path
compiled in place (oracle/_ref/libsdddst_ref.so, built by `make -C oracle ref`
where the reference sources exist).  The reference ships no tests, golden
vectors or fixtures of its own, so these outputs of the reference itself are
the pins of the oracle restatement and of the CUDA path.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from sdddst_b200 import workloads  # noqa: E402

CASES = {
    # name: (n, seed, p, cutoff multiplier, prec, stress kind, stress value, steps)
    "n64_zero": (64, 10, 0, 0.5, 1e-6, 0, 0.0, 6),
    "n96_pd8_const": (96, 11, 8, 1.0, 1e-7, 3, 0.01, 4),
    "n128_m1_zero": (128, 12, 0, 1.0, 1e-6, 0, 0.0, 4),
}


def field_case():
    rng = np.random.default_rng(20)
    dx = rng.uniform(-0.5, 0.5, 3000)
    dy = rng.uniform(-0.5, 0.5, 3000)
    dx[:300] *= 1e-3  # reference Taylor branch (r^2 <= 1e-6)
    dy[:300] *= 1e-3
    dx[300:400] = -dx[300:400] * 0  # dx = 0 exactly
    dx[400:500] = 0.5 - 1e-12      # near the wrap edge
    xy = ref.field(0, dx, dy, "ref")
    xy_dx = ref.field(1, dx, dy, "ref")
    np.savez_compressed(os.path.join(HERE, "field.npz"), dx=dx, dy=dy, xy=xy, xy_dx=xy_dx)


def sim_case(name, n, seed, p, m, prec, sk, sv, steps):
    xyb, pd = workloads.dislocations(n, seed, p)
    prm = ref.params(cutoff_multiplier=m, prec=prec, step_size=1e-6, stress_kind=sk, stress_value=sv,
                     pd_scaling=p > 0)
    s = ref.Sim(xyb, pd, prm, "ref")
    v, tol = s.speeds(xyb)
    h = 2e-6
    Ap, Ai, Ax, dvec = s.jacobian(h, xyb)
    traj_x, traj_sc, acc = [], [], []
    for _ in range(steps):
        acc.append(s.step())
        traj_x.append(s.config(0)[:, 0].copy())
        sc = s.scalars()
        traj_sc.append([sc[k] for k in ref.SCALAR_NAMES])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), xyb=xyb, pd=pd, v=v, tol=tol, h=h, Ap=Ap, Ai=Ai,
                        Ax=Ax, dvec=dvec, traj_x=np.array(traj_x), traj_scalars=np.array(traj_sc),
                        accepted=np.array(acc), params=np.array([n, seed, p, m, prec, sk, sv, steps]))


if __name__ == "__main__":
    if not ref.available("ref"):
        sys.exit("oracle/_ref/libsdddst_ref.so is missing: run `make -C oracle ref` first")
    field_case()
    for name, args in CASES.items():
        sim_case(name, *args)
    print("written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
