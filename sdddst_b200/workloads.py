"""Seeded synthetic workloads for the implicit-step hot path.

The reference ships no configurations, fixtures or benchmark inputs; these
generators are frozen so that the CUDA path, the CPU oracle and the bench all
read identical states.  Every generator uses ``numpy.random.default_rng(seed)``
(PCG64) and draws, in this order:

* dislocation positions ``rng.uniform(-0.5, 0.5, (N, 2))`` (column 0 = x,
  column 1 = y), i.e. the reference's simulation cell [-0.5, 0.5)^2
  (the reference's README.md, "Configuration files");
* Burgers signs ``rng.permutation([+1]*(N//2) + [-1]*(N - N//2))``;
* point defects ``rng.uniform(-0.5, 0.5, (P, 2))``, after the dislocations.

States are returned as an (N, 3) float64 array of (x, y, b) rows -- the
reference's ``Dislocation{x, y, b}`` layout (include/dislocation.h:27-31) and
its ``.dconf`` text format (src/simulation_data.cpp:119-161).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


def dislocations(n: int, seed: int, p: int = 0):
    """Return ``(xyb, pd)``: an (n, 3) dislocation array and a (p, 2) array of
    point defects, drawn from ``default_rng(seed)`` as described above."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n, 2))
    signs = rng.permutation(np.array([1.0] * (n // 2) + [-1.0] * (n - n // 2)))
    xyb = np.empty((n, 3), dtype=np.float64)
    xyb[:, 0] = pos[:, 0]
    xyb[:, 1] = pos[:, 1]
    xyb[:, 2] = signs
    pd = rng.uniform(-0.5, 0.5, (p, 2)) if p > 0 else np.zeros((0, 2))
    return xyb, np.ascontiguousarray(pd, dtype=np.float64)


def batch_sizes(count: int, seed: int, lo: int = 64, hi: int = 2048):
    """Per-realisation dislocation counts ``rng.integers(lo, hi + 1, count)``."""
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, count)


def batch(count: int, seed: int, lo: int = 64, hi: int = 2048):
    """``count`` independent realisations with uneven N: the sizes come from
    ``batch_sizes(count, seed)``; realisation k uses seed ``seed*100003 + k``
    for its own positions and signs."""
    sizes = batch_sizes(count, seed, lo, hi)
    return [dislocations(int(n), seed * 100003 + k)[0] for k, n in enumerate(sizes)]


def write_dconf(path: str, xyb: np.ndarray) -> None:
    """Write a dislocation file in the reference's format: one ``x y b`` line
    per dislocation, scientific with 16 digits (simulation_data.cpp:152-161),
    which round-trips doubles exactly."""
    with open(path, "w") as f:
        for x, y, b in xyb:
            f.write(f"{x:.16e} {y:.16e} {b:.16e}\n")


def write_pdconf(path: str, pd: np.ndarray) -> None:
    """Point-defect file: ``x y`` per line (simulation_data.cpp:192-201)."""
    with open(path, "w") as f:
        for x, y in pd:
            f.write(f"{x:.16e} {y:.16e}\n")


def read_dconf(path: str) -> np.ndarray:
    """Read ``x y b`` triplets (simulation_data.cpp:119-150)."""
    data = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return np.ascontiguousarray(data.reshape(-1, 3))


def read_pdconf(path: str) -> np.ndarray:
    data = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return np.ascontiguousarray(data.reshape(-1, 2))


@dataclasses.dataclass(frozen=True)
class Workload:
    """One named run: sizes, seed and the scalar parameters of the step."""
    name: str
    n: int
    seed: int
    cutoff_multiplier: float
    prec: float
    p: int = 0
    stress_kind: int = 0          # 0 zero, 1 fixed-rate, 2 spring, 3 constant
    stress_value: float = 0.0
    step_size: float = 1e-6       # the CLI's --initial-stepsize default
    steps: int = 100
    pd_scaling: bool = False      # A *= 1/sqrt(N), KASQR *= N (CLI with a point-defect file)

    def state(self):
        return dislocations(self.n, self.seed, self.p)


# The five runs the hot path is specified on (sizes, seeds and parameters).
SMALL_256 = Workload("n256_m0.5_zero_stress", 256, 0, 0.5, 1e-6, steps=200)
PD_4096 = Workload("n4096_pd256_const0.01_m1.0", 4096, 1, 1.0, 1e-7, p=256,
                   stress_kind=3, stress_value=0.01, steps=100, pd_scaling=True)
# No precision is stated for the two largest runs: they use the CLI default
# --position-precision 1e-5 (project_parser.cpp:63).
MIXED_16384 = Workload("n16384_m1.0_mixed", 16384, 2, 1.0, 1e-5, steps=10)
LARGE_32768 = Workload("n32768_m2.0", 32768, 4, 2.0, 1e-5, steps=10)
BATCH_SEED = 3
BATCH_COUNT = 512
BATCH_M = 0.5
