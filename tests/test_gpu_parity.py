"""GPU parity of the CUDA path against the oracle, through the C ABI.

The oracle is the C restatement (oracle/sdddst_oracle.c), itself pinned
bit-for-bit to the reference (tests/test_oracle.py); the committed golden
fixtures of the reference are checked directly too.

Tolerances (FP64 plain path):
  * velocities: 1e-10 relative in the max norm, |dv_i| <= 1e-10 * max_j |v_j|
    for every i (the device sums pairs in a different order and evaluates the
    field with a shared exp and exact near-field identities instead of
    per-image cosh and a Taylor branch).  The bar is normwise, not
    element-wise: a velocity is a sum of O(N) terms of both signs, and where
    they cancel |v_i| is far below the terms it is made of, so no summation
    order reproduces it to 1e-10 of itself;
  * tolerances: bit-exact without point defects (same r^2 arithmetic);
  * Jacobian: same sparsity pattern, |dJ_ij| <= 1e-10 * max|J offdiag|;
  * positions after a teacher-forced step: 1e-10 relative, error ratio 1e-6
    relative (it divides a ~1e-6 position difference by a ~1e-12 tolerance),
    identical accept/reject decisions and step sizes to 1e-6 relative.
"""
import os

import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def make_pair(n, seed, m, prec, p=0, sk=0, sv=0.0, step=1e-6, rate=0.0, spring=1.0, strain=False, **kw):
    """The oracle and a CUDA engine on the same seeded configuration and
    parameters (stress protocol: sk kind, sv constant value, rate for the
    fixed-rate and spring protocols, spring constant, strain bookkeeping)."""
    from sdddst_b200 import capi
    xyb, pd = workloads.dislocations(n, seed, p)
    rp = ref.params(cutoff_multiplier=m, prec=prec, step_size=step, stress_kind=sk, stress_value=sv,
                    stress_rate=rate, spring_constant=spring, calculate_strain=strain, pd_scaling=p > 0)
    oracle = ref.Sim(xyb, pd if p else None, rp, "port")
    prm = capi.cli_params(n, m, prec, step_size=step, p=p, pd_scaling=p > 0, stress_kind=sk, stress_value=sv,
                          stress_rate=rate, spring_constant=spring, calculate_strain=int(strain), **kw)
    eng = capi.Engine(prm, xyb, pd if p else None)
    return xyb, pd, oracle, eng


def assert_speeds_close(v, v_ref):
    """1e-10 relative in the max norm (see the module docstring)."""
    scale = np.abs(v_ref).max()
    err = np.abs(v - v_ref)
    assert np.all(err <= 1e-10 * scale), (err.max() / scale, scale)


@pytest.mark.parametrize("n,seed,m,p,sk,sv", [(256, 0, 0.5, 0, 0, 0.0), (1000, 5, 1.0, 64, 3, 0.01),
                                              (4096, 1, 1.0, 256, 3, 0.01)])
def test_speeds_match_oracle(engine_lib, port_lib, n, seed, m, p, sk, sv):
    xyb, pd, o, e = make_pair(n, seed, m, 1e-6, p, sk, sv)
    for stype in (0, 2):
        v_ref, tol_ref = o.speeds(xyb, 0.0, stype)
        v, tol = e.speeds(xyb, 0.0, stype)
        assert_speeds_close(v, v_ref)
        if p == 0:
            assert np.array_equal(tol, tol_ref)
        else:
            assert np.allclose(tol, tol_ref, rtol=1e-9, atol=0)


@pytest.mark.parametrize("name", ["n64_zero", "n96_pd8_const", "n128_m1_zero"])
def test_speeds_and_jacobian_match_golden(engine_lib, name):
    from sdddst_b200 import capi
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    n, seed, p, m, prec, sk, sv, steps = g["params"]
    n, p = int(n), int(p)
    prm = capi.cli_params(n, m, prec, step_size=1e-6, p=p, pd_scaling=p > 0, stress_kind=int(sk), stress_value=sv)
    e = capi.Engine(prm, g["xyb"], g["pd"] if p else None)
    v, tol = e.speeds(g["xyb"])
    assert_speeds_close(v, g["v"])
    _compare_jacobian(e, float(g["h"]), g["xyb"], g["Ap"], g["Ai"], g["Ax"], g["dvec"], n)


def _dense_from_csc(Ap, Ai, Ax, n):
    return ref.csc_to_dense(Ap, Ai, Ax, n)


def _compare_jacobian(e, h, xyb, Ap, Ai, Ax, dvec_ref, n):
    rp, col, val, d = e.jacobian(h, xyb)
    J = np.zeros((n, n))
    pat = np.zeros((n, n), dtype=bool)
    for i in range(n):
        for q in range(rp[i], rp[i + 1]):
            J[i, col[q]] += val[q]
            pat[i, col[q]] = True
    Jr = _dense_from_csc(Ap, Ai, Ax, n)
    pr = np.zeros((n, n), dtype=bool)
    for j in range(n):
        for q in range(Ap[j], Ap[j + 1]):
            pr[Ai[q], j] = True
    pr = pr | pr.T
    assert np.array_equal(pat, pr), "sparsity pattern differs"
    off = ~np.eye(n, dtype=bool)
    scale = np.abs(Jr[off]).max() if np.any(off & pr) else 1.0
    assert np.abs(J - Jr).max() <= 1e-10 * max(scale, 1.0)
    assert np.allclose(d, dvec_ref, rtol=1e-9, atol=1e-14)


@pytest.mark.parametrize("n,seed,m,p,h", [(256, 0, 0.5, 0, 3e-6), (600, 3, 1.0, 32, 1e-5)])
def test_jacobian_matches_oracle(engine_lib, port_lib, n, seed, m, p, h):
    xyb, pd, o, e = make_pair(n, seed, m, 1e-6, p, 3 if p else 0, 0.01 if p else 0.0)
    Ap, Ai, Ax, d = o.jacobian(h, xyb)
    _compare_jacobian(e, h, xyb, Ap, Ai, Ax, d, n)


def test_jacobian_clustered_cells(engine_lib, port_lib):
    """A cluster of 4200 dislocations in one 0.04 x 0.04 square among 1800
    spread ones (N=6000, cutoff multiplier 1, 10 x 10 cells): the four
    neighbour blocks holding the whole cluster exceed the shared-memory stage
    of the assembly (4096 candidates) and walk global memory with the FP64
    test, the others are staged with the FP32 prefilter; the CSR is the
    oracle's either way (pattern exact, values 1e-10)."""
    import scipy.sparse as sp
    from sdddst_b200 import capi
    rng = np.random.default_rng(8)
    n, m, h = 6000, 1.0, 1e-6
    pos = np.concatenate([rng.uniform(-0.5, 0.5, (1800, 2)), 0.1 + rng.uniform(-0.02, 0.02, (4200, 2))])
    b = rng.permutation(np.r_[np.ones(n // 2), -np.ones(n // 2)])
    xyb = np.column_stack([pos, b])
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=1e-6), "port")
    e = capi.Engine(capi.cli_params(n, m, 1e-6), xyb)
    Ap, Ai, Ax, d_ref = o.jacobian(h, xyb)
    rp, col, val, d = e.jacobian(h, xyb)
    J = sp.csr_matrix((val, col, rp), shape=(n, n)).tocoo()
    Jr = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n)).tocsr()
    pat = sp.csr_matrix((np.ones(J.nnz), (J.row, J.col)), shape=(n, n))
    pr = Jr.copy()
    pr.data[:] = 1.0
    pr = ((pr + pr.T) > 0).astype(float)
    assert (pat != pr).nnz == 0, "sparsity pattern differs"
    diff = abs(J.tocsr() - Jr)
    off = sp.triu(abs(Jr), 1)
    assert diff.max() <= 1e-10 * max(off.max(), 1.0)
    # d_i depends on the row sum G_ii, whose rounding grows with the row's
    # cancellation kappa_i = sum_j |J_ij| / |J_ii - 1| (above 1e4 inside the
    # cluster, where terms of size 1e6 cancel): the bound scales with it
    jd = Jr.diagonal()
    rowabs = np.asarray(abs(Jr - sp.diags(jd)).sum(1)).ravel()
    kappa = np.maximum(rowabs / np.maximum(np.abs(jd - 1.0), 1e-300), 1.0)
    assert np.all(np.abs(d - d_ref) <= 1e-14 + 1e-9 * kappa * np.abs(d_ref))


def test_solve_matches_dense(engine_lib, port_lib):
    n = 800
    xyb, pd, o, e = make_pair(n, 4, 1.0, 1e-6)
    h = 2e-5
    Ap, Ai, Ax, d = o.jacobian(h, xyb)
    J = ref.csc_to_dense(Ap, Ai, Ax, n)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(n) * 1e-4
    x, iters = e.solve(h, xyb, b)
    x_ref = np.linalg.solve(J, b)
    assert iters > 0
    # residual at the solver's target; the solution to cond(J) times that
    assert np.linalg.norm(J @ x - b) <= 1e-11 * np.linalg.norm(b)
    cond = np.linalg.cond(J)
    assert np.abs(x - x_ref).max() <= 1e-13 * cond * np.abs(x_ref).max()


def _teacher_forced(n, seed, m, prec, p=0, sk=0, sv=0.0, steps=12, warm=0, **kw):
    """`steps` attempts, each started on both sides from the oracle's accepted
    state.  warm > 0: the engine first runs `warm` attempts alone (the step
    size leaves the initial transient), and the oracle starts from the
    engine's state after them."""
    xyb, pd, o, e = make_pair(n, seed, m, prec, p, sk, sv, **kw)
    first = True
    worst = 0.0
    decisions = 0
    if warm:
        for _ in range(warm):
            e.step()
        sc = e.scalars()
        o.set_state(e.config(0), sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
        first = False
    accepted = 0
    for k in range(steps):
        x = o.config(0)
        sc = o.scalars()
        h = sc["step_size"]
        e.set_state(x, h, sc["sim_time"], sc["energy"], sc["strain"], first)
        if not first:
            o.set_state(x, h, sc["sim_time"], sc["energy"], sc["strain"], False)
        first = False
        a_ref = o.step()
        a = e.step()
        so, se = o.scalars(), e.scalars()
        assert a == a_ref, (k, so, se)
        decisions += 1
        accepted += a
        for which in (1, 2, 3):
            xr = o.config(which)[:, 0]
            xd = e.config(which)[:, 0]
            worst = max(worst, np.abs(xd - xr).max())
            assert np.abs(xd - xr).max() <= 1e-10 * max(1.0, np.abs(xr).max()), (k, which)
        assert np.isclose(se["max_error_ratio_sqr"], so["max_error_ratio_sqr"], rtol=1e-6, atol=1e-12), (k, so, se)
        assert np.isclose(se["step_size"], so["step_size"], rtol=1e-6), k
        assert np.isclose(se["energy"], so["energy"], rtol=1e-9, atol=1e-300), k
        assert np.allclose(e.vector(6), o.vector(6), rtol=1e-9, atol=0)
        assert np.isclose(se["stress"], so["stress"], rtol=1e-12, atol=0), k
        assert np.isclose(se["strain"], so["strain"], rtol=1e-9, atol=1e-18), k
    _teacher_forced.accepted = accepted
    return worst, decisions


def test_step_teacher_forced_small(engine_lib, port_lib):
    worst, k = _teacher_forced(256, 0, 0.5, 1e-6, steps=16)
    assert k == 16


def test_step_teacher_forced_defects_constant_stress(engine_lib, port_lib):
    worst, k = _teacher_forced(600, 1, 1.0, 1e-7, p=40, sk=3, sv=0.01, steps=5)
    assert k == 5


def test_free_running_trajectory_small(engine_lib, port_lib):
    """200 accepted steps of the N=256 workload, free running on both sides;
    per-step positions, error ratio and energy are compared while the two
    trajectories take the same accept/reject decisions."""
    w = workloads.SMALL_256
    xyb, _ = w.state()
    from sdddst_b200 import capi
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=w.cutoff_multiplier, prec=w.prec, step_size=w.step_size), "port")
    e = capi.Engine(capi.cli_params(w.n, w.cutoff_multiplier, w.prec, step_size=w.step_size), xyb)
    acc = 0
    attempts = 0
    while acc < w.steps and attempts < 600:
        a_ref = o.step()
        a = e.step()
        attempts += 1
        assert a == a_ref, attempts
        acc += a
        so, se = o.scalars(), e.scalars()
        xr, xd = o.config(0)[:, 0], e.config(0)[:, 0]
        assert np.abs(xd - xr).max() <= 1e-9, attempts
        assert np.isclose(se["max_error_ratio_sqr"], so["max_error_ratio_sqr"], rtol=1e-5, atol=1e-12)
        assert np.isclose(se["energy"], so["energy"], rtol=1e-8)
    assert acc == w.steps


def test_fp32_pairsum_accuracy(engine_lib, port_lib):
    """Mixed precision: FP32 pair terms with FP64 accumulation against the
    FP64 oracle (reported error, bounded here)."""
    from sdddst_b200 import capi
    n = 4096
    xyb, _ = workloads.dislocations(n, 2)
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=1.0, prec=1e-5), "port")
    v_ref, _ = o.speeds(xyb)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-5, pairsum=capi.PAIRSUM_FP32), xyb)
    v, _ = e.speeds(xyb)
    rel = np.abs(v - v_ref).max() / np.abs(v_ref).max()
    assert rel < 1e-5, rel


def test_fp32_pairsum_close_and_boundary_pairs(engine_lib, port_lib):
    """Mixed precision on the pairs that are hardest for FP32 terms:
    separations from 1e-6 to 1e-2 and pairs straddling the periodic boundary
    in x and in y.  Every velocity is within 2e-6 of the sum of the magnitudes
    of its terms (FP32 terms carry about 1e-7 relative error; 16-term FP32
    partial sums add at most 15 roundings)."""
    from sdddst_b200 import capi
    rng = np.random.default_rng(21)
    m = 192
    base = rng.uniform(-0.5, 0.5, (m, 2))
    r = 10.0 ** rng.uniform(-6, -2, m)
    ang = rng.uniform(0, 2 * np.pi, m)
    close = base + np.stack([r * np.cos(ang), r * np.sin(ang)], 1)
    edge = rng.uniform(-0.5, 0.5, (128, 2))
    edge[:64, 0] = 0.5 - 10.0 ** rng.uniform(-6, -3, 64) * rng.choice([1.0, 2.0], 64)
    edge[64:, 1] = -0.5 + 10.0 ** rng.uniform(-6, -3, 64)
    edge2 = edge.copy()
    edge2[:64, 0] -= 1.0 - 10.0 ** rng.uniform(-6, -4, 64)
    edge2[64:, 1] += 1.0 - 10.0 ** rng.uniform(-6, -4, 64)
    pos = np.concatenate([base, close, edge, edge2])
    pos -= np.rint(pos)
    pos[pos >= 0.5] -= 1.0
    n = len(pos)
    b = rng.permutation(np.r_[np.ones(n // 2), -np.ones(n - n // 2)])
    xyb = np.column_stack([pos, b])
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=1.0, prec=1e-5), "port")
    v_ref, _ = o.speeds(xyb)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-5, pairsum=capi.PAIRSUM_FP32), xyb)
    v, _ = e.speeds(xyb)
    dx = pos[:, None, 0] - pos[None, :, 0]
    dy = pos[:, None, 1] - pos[None, :, 1]
    dx -= np.rint(dx)
    dy -= np.rint(dy)
    off = ~np.eye(n, dtype=bool)
    mag = np.zeros((n, n))
    mag[off] = np.abs(ref.field(0, dx[off], dy[off], "port"))
    scale = mag.sum(1)
    err = (np.abs(v - v_ref) / scale).max()
    assert err <= 2e-6, err


def test_mixed_jacobian_close_to_oracle(engine_lib, port_lib):
    """Mixed path: FP32 dtau/dx and FP32 storage of G; J within FP32
    accuracy of the oracle's (the pattern is the same test in FP64)."""
    from sdddst_b200 import capi
    n, h = 600, 1e-5
    xyb, pd, o, _ = make_pair(n, 3, 1.0, 1e-6)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-6, pairsum=capi.PAIRSUM_FP32), xyb)
    Ap, Ai, Ax, d = o.jacobian(h, xyb)
    rp, col, val, dd = e.jacobian(h, xyb)
    J = np.zeros((n, n))
    for i in range(n):
        for q in range(rp[i], rp[i + 1]):
            J[i, col[q]] += val[q]
    Jr = ref.csc_to_dense(Ap, Ai, Ax, n)
    off = ~np.eye(n, dtype=bool)
    assert np.abs(J - Jr)[off].max() <= 2e-5 * np.abs(Jr[off]).max()
    assert np.abs(np.diag(J) - np.diag(Jr)).max() <= 2e-5 * np.abs(np.diag(Jr)).max()


def test_step_teacher_forced_config2_scale(engine_lib, port_lib):
    """The plain-method workload at scale: N=4096 + 256 point defects
    (seed 1), constant external stress 0.01, cutoff multiplier 1, precision
    1e-7, device sparse LU.  Five attempts teacher-forced against the oracle
    after the step size has left the initial transient (12 attempts of the
    engine alone): stage positions within 1e-10, identical decisions, error
    ratio, step size and energy as in the smaller cases."""
    from sdddst_b200 import capi
    worst, k = _teacher_forced(4096, 1, 1.0, 1e-7, p=256, sk=3, sv=0.01, steps=5, warm=12,
                               solver=capi.SOLVER_DIRECT)
    assert k == 5 and _teacher_forced.accepted >= 2, _teacher_forced.accepted


def test_step_teacher_forced_config2_gmres(engine_lib, port_lib):
    """The same workload with the cluster-preconditioned GMRES solver."""
    worst, k = _teacher_forced(4096, 1, 1.0, 1e-7, p=256, sk=3, sv=0.01, steps=3, warm=12)
    assert k == 3


@pytest.mark.parametrize("sk,rate,spring", [(1, 2.0e4, 1.0), (2, 5.0e5, 20.0)])
def test_step_teacher_forced_stress_protocols(engine_lib, port_lib, sk, rate, spring):
    """FixedRateProtocol (fixed_rate_protocol.cpp:39-57: tau = t * rate per
    stage) and SpringProtocol (spring_protocol.cpp:33-54: tau = k (t rate -
    strain), clamped at 0, with the strain of the stage's configuration fed
    back, simulation.cpp:154,180,544) teacher-forced against the oracle with
    strain bookkeeping on: stage positions, decisions, stress and strain.
    The rate makes the external stress comparable with the internal stresses
    within the run."""
    worst, k = _teacher_forced(600, 13, 1.0, 1e-6, sk=sk, rate=rate, spring=spring, strain=True, steps=10, warm=4)
    assert k == 10 and _teacher_forced.accepted >= 3


def test_free_running_stress_protocols_reach_stress(engine_lib, port_lib):
    """Free-running fixed-rate and spring runs of 30 attempts against the
    oracle: the stress of the accepted state grows with the simulated time
    (spring: by k (t rate - strain)), and the two sides stay together."""
    from sdddst_b200 import capi
    for sk, rate, spring in ((1, 2.0e4, 1.0), (2, 5.0e5, 20.0)):
        xyb, pd, o, e = make_pair(400, 14, 1.0, 1e-6, sk=sk, rate=rate, spring=spring, strain=True)
        for k in range(30):
            assert e.step() == o.step(), (sk, k)
            so, se = o.scalars(), e.scalars()
            assert np.abs(e.config(0)[:, 0] - o.config(0)[:, 0]).max() <= 1e-9, (sk, k)
            assert np.isclose(se["stress"], so["stress"], rtol=1e-9, atol=1e-300), (sk, k)
            assert np.isclose(se["strain"], so["strain"], rtol=1e-7, atol=1e-18), (sk, k)
        assert se["stress"] > 0.0, (sk, se)


def test_order_parameter_matches_oracle(engine_lib, port_lib):
    """calculateOrderParameter (simulation.cpp:407-415): sum_i b_i v_i of the
    accepted configuration over the step's speed vector, after teacher-forced
    steps; the speed vectors themselves within the velocity bar."""
    xyb, pd, o, e = make_pair(500, 15, 1.0, 1e-6)
    for k in range(6):
        x, sc = o.config(0), o.scalars()
        e.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], k == 0)
        if k:
            o.set_state(x, sc["step_size"], sc["sim_time"], sc["energy"], sc["strain"], False)
        assert e.step() == o.step(), k
        for which in (2, 3):  # speed, speed2
            assert_speeds_close(e.vector(which), o.vector(which))
        b = o.config(0)[:, 2]
        op_ref = float(np.dot(b, o.vector(2)))
        op = float(np.dot(e.config(0)[:, 2], e.vector(2)))
        assert abs(op - op_ref) <= 1e-10 * np.abs(b * o.vector(2)).sum(), (k, op, op_ref)


def test_jacobian_multiblock_scan_n20001(engine_lib, port_lib):
    """N = 20001 (above the one-block scan's 16384 entries and not a multiple
    of its 2048-entry chunks): the row pointers, columns and values of the
    assembled CSR against the oracle (pattern exact, values 1e-10), and a
    solve through the preconditioner whose pattern counts use the same
    multi-block scan."""
    import scipy.sparse as sp
    n, h = 20001, 2e-6
    xyb, pd, o, e = make_pair(n, 17, 1.0, 1e-6)
    Ap, Ai, Ax, d_ref = o.jacobian(h, xyb)
    rp, col, val, d = e.jacobian(h, xyb)
    J = sp.csr_matrix((val, col, rp), shape=(n, n))
    Jr = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n)).tocsr()
    pr = Jr.copy()
    pr.data[:] = 1.0
    pr = ((pr + pr.T) > 0).astype(np.int8).tocsr()
    pat = sp.csr_matrix((np.ones(len(col), dtype=np.int8), col, rp), shape=(n, n))
    assert np.array_equal(np.diff(rp), np.diff(pr.indptr)), "row counts differ"
    assert (pat != pr).nnz == 0, "sparsity pattern differs"
    off = sp.triu(abs(Jr), 1)
    assert abs(J - Jr).max() <= 1e-10 * max(off.max(), 1.0)
    rhs = np.random.default_rng(3).standard_normal(n) * 1e-4
    x, iters = e.solve(h, xyb, rhs)
    assert np.linalg.norm(J @ x - rhs) <= 1e-12 * np.linalg.norm(rhs)


@pytest.mark.parametrize("m", [1000, 2048, 2049, 16385, 20001, 131072, 131073, 300001])
def test_scan_routes_match_cumsum(engine_lib, m):
    """The exclusive scan behind the CSR row pointers and the preconditioner's
    offsets, on each of its routes (one block up to 2048 entries, one launch
    of self-offsetting chunks up to 64 x 2048, three launches above), against
    numpy's cumulative sum."""
    import ctypes as C
    import torch
    from sdddst_b200 import capi
    xyb, _ = workloads.dislocations(256, 0)
    e = capi.Engine(capi.cli_params(256, 0.5, 1e-6), xyb)
    vals = np.random.default_rng(m).integers(0, 700, m).astype(np.int32)
    src = torch.tensor(vals, device="cuda")
    dst = torch.full((m + 1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    fn = e.lib.sdddst_internal_scan
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    fn.restype = C.c_int
    assert fn(e.h, src.data_ptr(), m, dst.data_ptr()) == 0
    want = np.concatenate([[0], np.cumsum(vals, dtype=np.int64)])
    assert np.array_equal(dst.cpu().numpy().astype(np.int64), want)
    e.close()


def test_solve_with_restarts_matches_dense(engine_lib, port_lib):
    """The device-resident GMRES with a restart length of 4 (several restart
    cycles: the true residual recomputed, the basis rebuilt) against a dense
    solve with the oracle's Jacobian, as test_solve_matches_dense."""
    n = 800
    xyb, pd, o, e = make_pair(n, 4, 1.0, 1e-6, gmres_restart=4)
    h = 2e-5
    Ap, Ai, Ax, d = o.jacobian(h, xyb)
    J = ref.csc_to_dense(Ap, Ai, Ax, n)
    b = np.random.default_rng(0).standard_normal(n) * 1e-4
    x, iters = e.solve(h, xyb, b)
    assert iters > 4
    assert np.linalg.norm(J @ x - b) <= 1e-11 * np.linalg.norm(b)
    x_ref = np.linalg.solve(J, b)
    assert np.abs(x - x_ref).max() <= 1e-13 * np.linalg.cond(J) * np.abs(x_ref).max()
