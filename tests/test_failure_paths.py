"""Failure paths of the engine, in forms that fault or hang no GPU: bad
inputs are refused on the host, solver stalls are made by a one-iteration
cap, and capacity is exceeded by a too-small caller buffer.

The reference detects none of these: a NaN or a coincident pair of
dislocations gives NaN velocities that it accepts as a step
(src/simulation.cpp:86-131, 516), the UMFPACK status is cast to void
(src/simulation.cpp:388-395), and the CSC buffers are sized up front.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads


def test_create_rejects_nonfinite_configuration_on_the_host(engine_lib):
    """NaN / Inf in the configuration or the point defects: refused by
    sdddst_ctx_create and sdddst_batch_create before any device work (runs
    without a GPU)."""
    from sdddst_b200 import capi
    xyb, pd = workloads.dislocations(64, 3, 4)
    for bad, where in ((np.nan, (5, 0)), (np.inf, (7, 1)), (-np.inf, (9, 2))):
        a = xyb.copy()
        a[where] = bad
        with pytest.raises(capi.EngineError) as ex:
            capi.Engine(capi.cli_params(64, 0.5, 1e-6), a)
        assert ex.value.rc == capi.ERR_NONFINITE and str(3 * where[0] + where[1]) in str(ex.value)
    p = pd.copy()
    p[2, 1] = np.nan
    with pytest.raises(capi.EngineError) as ex:
        capi.Engine(capi.cli_params(64, 0.5, 1e-6, p=4, pd_scaling=True), xyb, p)
    assert ex.value.rc == capi.ERR_NONFINITE
    a = xyb.copy()
    a[11, 0] = np.nan
    with pytest.raises(capi.EngineError) as ex:
        capi.Batch(capi.default_params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6), [xyb, a])
    assert ex.value.rc == capi.ERR_NONFINITE


@pytest.mark.gpu
def test_set_state_and_upload_reject_nonfinite_and_context_survives(engine_lib, port_lib):
    from sdddst_b200 import capi
    n = 256
    xyb, _ = workloads.dislocations(n, 0)
    e = capi.Engine(capi.cli_params(n, 0.5, 1e-6), xyb)
    bad = xyb.copy()
    bad[17, 1] = np.nan
    with pytest.raises(capi.EngineError) as ex:
        e.set_state(bad, 1e-6, first_step=True)
    assert ex.value.rc == capi.ERR_NONFINITE
    xs = np.ascontiguousarray(xyb[:, 0].copy())
    xs[3] = np.inf
    with pytest.raises(capi.EngineError) as ex:
        e.upload_positions(xs)
    assert ex.value.rc == capi.ERR_NONFINITE
    # nothing reached the device: the context steps exactly like the oracle
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6), "port")
    for k in range(4):
        assert e.step() == o.step(), k
        assert np.abs(e.config(0)[:, 0] - o.config(0)[:, 0]).max() <= 1e-10


@pytest.mark.gpu
def test_coincident_dislocations(engine_lib, port_lib):
    """Two pairs of dislocations at identical positions (one of opposite
    signs, one of equal signs).  The tolerance takes the EPS path of
    PrecisionHandler::updateTolerance (precision_handler.cpp:75-81) exactly as
    in the reference; the velocities of every other dislocation match the
    oracle; the coincident ones are non-finite on both sides (the field is
    singular at zero separation).  The reference then steps on with NaN
    positions; the engine stops the step with SDDDST_ERR_NONFINITE."""
    from sdddst_b200 import capi
    n = 64
    xyb, _ = workloads.dislocations(n, 3)
    xyb[5, :2] = xyb[9, :2]
    xyb[5, 2], xyb[9, 2] = 1.0, -1.0
    xyb[20, :2] = xyb[21, :2]
    xyb[20, 2], xyb[21, 2] = 1.0, 1.0
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6), "port")
    e = capi.Engine(capi.cli_params(n, 0.5, 1e-6), xyb)
    v_ref, tol_ref = o.speeds(xyb)
    v, tol = e.speeds(xyb)
    assert np.array_equal(tol, tol_ref)
    coincident = np.array([5, 9, 20, 21])
    assert np.all(tol[coincident] == 1e-12)
    fin = np.isfinite(v_ref)
    assert not fin[coincident].any() and fin.sum() == n - 4
    assert np.array_equal(np.isfinite(v), fin)
    assert np.all(np.abs(v[fin] - v_ref[fin]) <= 1e-10 * np.abs(v_ref[fin]).max())
    with pytest.raises(capi.EngineError) as ex:
        e.step()
    assert ex.value.rc == capi.ERR_NONFINITE


@pytest.mark.gpu
def test_cluster_gmres_stall_rebuilds_then_reports(engine_lib):
    """A one-iteration cap (no preconditioned solve of this system reaches a
    1e-13 residual in one iteration): the cluster-preconditioned GMRES stalls,
    the preconditioner is rebuilt twice with a lower coupling threshold, and
    the solve reports SDDDST_ERR_SOLVER.  With the cap lifted the same context
    solves to the residual target."""
    import scipy.sparse as sp
    from sdddst_b200 import capi
    n, h = 800, 2e-5
    xyb, _ = workloads.dislocations(n, 4)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-6, max_iters=1), xyb)
    rhs = np.random.default_rng(6).standard_normal(n) * 1e-4
    with pytest.raises(capi.EngineError) as ex:
        e.solve(h, xyb, rhs)
    assert ex.value.rc == capi.ERR_SOLVER
    assert e.solver_recoveries()[0] == 2
    e.update_params(max_iters=300)
    x, iters = e.solve(h, xyb, rhs)
    rp, col, val, _ = e.jacobian(h, xyb)
    J = sp.csr_matrix((val, col, rp), shape=(n, n))
    assert iters > 1 and np.linalg.norm(J @ x - rhs) <= 1e-12 * np.linalg.norm(rhs)


@pytest.mark.gpu
def test_learned_stall_falls_back_to_sparse_lu(engine_lib, port_lib):
    """The learned-preconditioned GMRES capped at one iteration stalls on
    every solve and falls back to the device sparse LU of the same matrix:
    the steps still match the oracle (teacher-forced, positions 1e-10,
    same decisions) and every solve is counted as a fallback."""
    from sdddst_b200 import capi
    n = 300
    xyb, _ = workloads.dislocations(n, 2)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-6, solver=capi.SOLVER_GMRES_LEARNED, max_iters=1), xyb)
    e.set_preconditioner_weights()
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=1.0, prec=1e-6, step_size=1e-6), "port")
    for k in range(5):
        x, sc = o.config(0), o.scalars()
        e.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], k == 0)
        if k:
            o.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
        assert e.step() == o.step(), k
        for which in (1, 2, 3):
            assert np.abs(e.config(which)[:, 0] - o.config(which)[:, 0]).max() <= 1e-10, (k, which)
    # every GMRES solve stalled and was redone by the LU; both count as solves
    solves, _ = e.solver_stats()
    fallbacks = e.solver_recoveries()[1]
    assert fallbacks >= 5 and solves == 2 * fallbacks, (fallbacks, solves)


@pytest.mark.gpu
def test_jacobian_capacity_reports_needed_size(engine_lib):
    """A caller buffer smaller than the pattern: SDDDST_ERR_CAPACITY with the
    entry count needed, then the export succeeds with exactly that size."""
    from sdddst_b200 import capi
    n = 500
    xyb, _ = workloads.dislocations(n, 4)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-6), xyb)
    lib = capi.load()
    a = np.ascontiguousarray(xyb.reshape(-1))
    rp = np.zeros(n + 1, dtype=np.int32)
    col = np.zeros(16, dtype=np.int32)
    val = np.zeros(16)
    d = np.zeros(n)
    nnz = C.c_long(0)
    rc = lib.sdddst_jacobian(e.h, 1e-6, a, rp, col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p),
                             d.ctypes.data_as(C.c_void_p), 16, C.byref(nnz))
    assert rc == capi.ERR_CAPACITY and nnz.value > 16
    rp2, col2, val2, _ = e.jacobian(1e-6, xyb)
    assert len(col2) == nnz.value == rp2[-1]


@pytest.mark.gpu
def test_pattern_growth_redoes_the_attempt(engine_lib, port_lib):
    """The cluster solver's attempts run without waiting for the device and
    check everything once at the end.  An engine whose Jacobian storage was
    sized for a uniform configuration is given a strongly clustered one (4200
    of 6000 dislocations in a 0.04 x 0.04 square): the first assembly of the
    attempt outgrows the storage, is guarded (no access past it), the storage
    grows, and the attempt is redone with waits.  The step still matches the
    oracle's (decision, stage positions within 1e-10)."""
    from sdddst_b200 import capi
    rng = np.random.default_rng(8)
    n, m = 6000, 1.0
    uniform, _ = workloads.dislocations(n, 9)
    e = capi.Engine(capi.cli_params(n, m, 1e-6), uniform)
    pos = np.concatenate([rng.uniform(-0.5, 0.5, (1800, 2)), 0.1 + rng.uniform(-0.02, 0.02, (4200, 2))])
    b = rng.permutation(np.r_[np.ones(n // 2), -np.ones(n // 2)])
    xyb = np.column_stack([pos, b])
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=1e-6, step_size=1e-9), "port")
    o.set_state(xyb, 1e-9, 0.0, 0.0, 0.0, False)
    e.set_state(xyb, 1e-9, 0.0, 0.0, 0.0, False)
    assert e.step() == o.step()
    for which in (1, 2, 3):
        assert np.abs(e.config(which)[:, 0] - o.config(which)[:, 0]).max() <= 1e-10, which
    assert e.solver_recoveries()[2] >= 1
