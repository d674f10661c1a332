"""GPU tests of the sparse LU solver (SDDDST_SOLVER_DIRECT), the device
drop-in for the reference's UMFPACK factorization and solve
(simulation.cpp:386-396).

The oracle's solve runs through a project LU shim (UMFPACK itself is not
available), so the linear solve is checked against the oracle's Jacobian
with dense LAPACK: residual at the solver's target against the device's
own Jacobian (relative 1e-12; the direct solve is refined to 1e-13); against
the oracle's Jacobian, which agrees with the device's to 1e-10 of the largest
off-diagonal, the residual and the solution within that measured matrix
perturbation (times cond(J) for the solution).
Trajectories are checked against the oracle exactly like the GMRES path.
"""
import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads

from test_gpu_parity import _teacher_forced, make_pair

pytestmark = pytest.mark.gpu


def _direct(**kw):
    from sdddst_b200 import capi
    return dict(solver=capi.SOLVER_DIRECT, **kw)


@pytest.mark.parametrize("n,seed,m,p,h", [(256, 0, 0.5, 0, 3e-6), (800, 4, 1.0, 0, 2e-5),
                                          (1000, 5, 1.0, 64, 1e-5), (700, 6, 1.0, 0, 3e-3),
                                          (300, 7, 3.0, 0, 1e-4)])
def test_direct_solve_matches_dense(engine_lib, port_lib, n, seed, m, p, h):
    """Includes a stiff step (h = 3e-3: h |G| >> 1 for close pairs) and a
    cutoff multiplier above sqrt(2N)/12 (every pair coupled: one dense
    front)."""
    xyb, pd, o, e = make_pair(n, seed, m, 1e-6, p, 3 if p else 0, 0.01 if p else 0.0, **_direct())
    Ap, Ai, Ax, d = o.jacobian(h, xyb)
    J = ref.csc_to_dense(Ap, Ai, Ax, n)
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(n) * 1e-4
    x, refinements = e.solve(h, xyb, b)
    assert refinements <= 3
    # against the matrix the device factored (its own export) ...
    rp, col, val, _ = e.jacobian(h, xyb)
    Jd = np.zeros((n, n))
    for i in range(n):
        Jd[i, col[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]]
    assert np.linalg.norm(Jd @ x - b) <= 1e-12 * np.linalg.norm(b)
    # ... and against the oracle's J: the two matrices agree to 1e-10 of the
    # largest off-diagonal, so the residual and the solution move by that
    # perturbation (measured here) on top of the solve's own error
    dJ = np.linalg.norm(J - Jd, 2)
    assert np.linalg.norm(J @ x - b) <= 1e-12 * np.linalg.norm(b) + 2.0 * dJ * np.linalg.norm(x)
    x_ref = np.linalg.solve(J, b)
    cond = np.linalg.cond(J)
    rel = dJ / np.linalg.norm(J, 2)
    assert np.abs(x - x_ref).max() <= (cond * (2.0 * rel + 1e-12) + 1e-12) * np.abs(x_ref).max()
    st = e.direct_stats()
    assert st["factorizations"] >= 1 and st["fronts"] >= 1 and st["lu_flops"] > 0
    if m >= np.sqrt(2 * n) / 12:
        assert st["fronts"] == 1


def test_direct_solve_config2_scale(engine_lib):
    """N=4096 with 256 point defects, cutoff multiplier 1 (the plain-method
    workload at scale): residual against the device's own Jacobian export."""
    import scipy.sparse as sp
    from sdddst_b200 import capi
    n, p = 4096, 256
    xyb, pd = workloads.dislocations(n, 1, p)
    prm = capi.cli_params(n, 1.0, 1e-7, p=p, pd_scaling=True, stress_kind=capi.STRESS_CONSTANT, stress_value=0.01,
                          solver=capi.SOLVER_DIRECT)
    e = capi.Engine(prm, xyb, pd)
    for h in (1e-6, 1e-4):
        rp, col, val, d = e.jacobian(h, xyb)
        J = sp.csr_matrix((val, col, rp), shape=(n, n))
        b = np.random.default_rng(1).standard_normal(n)
        x, _ = e.solve(h, xyb, b)
        assert np.linalg.norm(J @ x - b) <= 1e-12 * np.linalg.norm(b)
    st = e.direct_stats()
    assert st["fronts"] > 3 and st["depth"] > 2


def test_direct_teacher_forced_small(engine_lib, port_lib):
    worst, k = _teacher_forced(256, 0, 0.5, 1e-6, steps=16, **_direct())
    assert k == 16


def test_direct_teacher_forced_defects_constant_stress(engine_lib, port_lib):
    worst, k = _teacher_forced(600, 1, 1.0, 1e-7, p=40, sk=3, sv=0.01, steps=5, **_direct())
    assert k == 5


def test_direct_free_running_small(engine_lib, port_lib):
    """The N=256 workload, 200 accepted steps with the sparse LU, free running
    against the oracle (same decisions, positions within 1e-9)."""
    from sdddst_b200 import capi
    w = workloads.SMALL_256
    xyb, _ = w.state()
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=w.cutoff_multiplier, prec=w.prec, step_size=w.step_size),
                "port")
    e = capi.Engine(capi.cli_params(w.n, w.cutoff_multiplier, w.prec, step_size=w.step_size,
                                    solver=capi.SOLVER_DIRECT), xyb)
    acc = attempts = 0
    while acc < w.steps and attempts < 600:
        a_ref = o.step()
        a = e.step()
        attempts += 1
        assert a == a_ref, attempts
        acc += a
        xr, xd = o.config(0)[:, 0], e.config(0)[:, 0]
        assert np.abs(xd - xr).max() <= 1e-9, attempts
        so, se = o.scalars(), e.scalars()
        assert np.isclose(se["max_error_ratio_sqr"], so["max_error_ratio_sqr"], rtol=1e-5, atol=1e-12)
        assert np.isclose(se["energy"], so["energy"], rtol=1e-8)
    assert acc == w.steps


def test_direct_matches_gmres_trajectory_config2(engine_lib):
    """N=4096 + 256 point defects, constant stress: the sparse LU and the
    cluster-preconditioned GMRES paths take the same decisions and stay
    within 1e-9 over 20 attempts (both solve to a 1e-13 residual)."""
    from sdddst_b200 import capi
    n, p = 4096, 256
    xyb, pd = workloads.dislocations(n, 1, p)
    engines = []
    for solver in (capi.SOLVER_DIRECT, capi.SOLVER_GMRES_CLUSTER):
        prm = capi.cli_params(n, 1.0, 1e-7, p=p, pd_scaling=True, stress_kind=capi.STRESS_CONSTANT,
                              stress_value=0.01, solver=solver)
        engines.append(capi.Engine(prm, xyb, pd))
    for k in range(20):
        a = [eng.step() for eng in engines]
        assert a[0] == a[1], k
        x0, x1 = engines[0].config(0)[:, 0], engines[1].config(0)[:, 0]
        assert np.abs(x0 - x1).max() <= 1e-9, k


@pytest.mark.parametrize("tensor_cores", [False, True])
def test_direct_mixed_solve_residual(engine_lib, tensor_cores, monkeypatch):
    """SDDDST_SOLVER_DIRECT_MIXED: FP32 fronts, FP64 refinement to the solver
    tolerance (relative residual 1e-12 against the device's own J), with the
    trailing updates on the CUDA cores (default) and on the tensor cores
    (compensated TF32, SDDDST_LU_TENSOR_CORES)."""
    import scipy.sparse as sp
    from sdddst_b200 import capi
    if tensor_cores:
        monkeypatch.setenv("SDDDST_LU_TENSOR_CORES", "1")
    else:
        monkeypatch.delenv("SDDDST_LU_TENSOR_CORES", raising=False)
    n, p = 4096, 256
    xyb, pd = workloads.dislocations(n, 1, p)
    prm = capi.cli_params(n, 1.0, 1e-7, p=p, pd_scaling=True, stress_kind=capi.STRESS_CONSTANT, stress_value=0.01,
                          solver=capi.SOLVER_DIRECT_MIXED)
    e = capi.Engine(prm, xyb, pd)
    for h in (1e-6, 1e-4):
        rp, col, val, d = e.jacobian(h, xyb)
        J = sp.csr_matrix((val, col, rp), shape=(n, n))
        b = np.random.default_rng(2).standard_normal(n)
        x, refinements = e.solve(h, xyb, b)
        assert refinements <= 10
        assert np.linalg.norm(J @ x - b) <= 1e-12 * np.linalg.norm(b)


def test_precision_workload_one_step_against_fp64(engine_lib):
    """The precision workload (N=16384, seed 2, cutoff multiplier 1): FP32 pair
    terms with FP64 accumulation, FP32 Jacobian values, FP32 LU with FP64
    refinement, against the plain FP64 path (FP64 pair sum, FP64 LU) one
    step from the same state: velocities within 1e-5 relative, positions
    within 1e-8 (the bar of the precision forms)."""
    from sdddst_b200 import capi
    n = 16384
    xyb, _ = workloads.dislocations(n, 2)
    common = dict(step_size=1e-6)
    e32 = capi.Engine(capi.cli_params(n, 1.0, 1e-5, pairsum=capi.PAIRSUM_FP32, solver=capi.SOLVER_DIRECT_MIXED,
                                      **common), xyb)
    e64 = capi.Engine(capi.cli_params(n, 1.0, 1e-5, pairsum=capi.PAIRSUM_FP64, solver=capi.SOLVER_DIRECT, **common),
                      xyb)
    v32, _ = e32.speeds(xyb)
    v64, _ = e64.speeds(xyb)
    assert np.abs(v32 - v64).max() <= 1e-5 * np.abs(v64).max()
    # the step size adapts first (the initial 1e-6 is rejected for close
    # pairs); then one step from the same accepted state on both paths
    accepted = 0
    for _ in range(12):
        accepted += e64.step()
        if accepted >= 3:
            break
    assert accepted >= 3
    for attempt in range(10):
        x, sc = e64.config(0), e64.scalars()
        for e in (e32, e64):
            e.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
        a32, a64 = e32.step(), e64.step()
        assert a32 == a64, (attempt, sc["step_size"], e32.scalars(), e64.scalars())
        if a64:
            for which in (1, 2, 3):
                assert np.abs(e32.config(which)[:, 0] - e64.config(which)[:, 0]).max() <= 1e-8, which
            return
    pytest.fail("no accepted step in 10 attempts")
