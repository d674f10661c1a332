"""The tabulated field (SDDDST_FIELD_TABULATED, host class
PeriodicShearStressELTE / PeriodicShearStressFieldELTEObject).

The reference's tabulated field has neither source nor data in the
reference, so the parity target is the analytic field within the
interpolation error: the tables hold the smooth remainder of the analytic
field after its image-free term, interpolated bicubically on a 1024 x 1024
grid; the image-free term is exact.  Bounds (measured errors are 2.4e-9 and
1.0e-8):
  * host field: |d tau_xy| r <= 1e-8 and |d tau_xy,x| r^2 <= 5e-8 over the
    cell, down to r = 1e-4;
  * device velocities: |dv_i| <= N * 1e-8 (every pair's term within 1e-8 of
    the analytic one at the separations of a random configuration);
  * device Jacobian: identical pattern, |dJ_ij| <= 5e-8 h / r^2 summed
    into the diagonal (checked as 1e-6 of the largest off-diagonal).
"""
import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads

from test_host_api import psc  # noqa: F401  (fixture)


def test_host_tabulated_matches_analytic(psc, port_lib):
    f = psc.PeriodicShearStressFieldELTEObject()
    f.setPWD(".")
    f.init()
    assert f.valid() and "ELTE" in f.name()
    d = psc.SimulationData("", "")
    d.tau = f
    tau = d.tau
    rng = np.random.default_rng(7)
    for lo, cnt in ((0.5, 3000), (0.01, 600), (1e-4, 200)):
        dx, dy = rng.uniform(-lo, lo, cnt), rng.uniform(-lo, lo, cnt)
        r = np.hypot(dx, dy)
        a, ad = ref.field(0, dx, dy, "port"), ref.field(1, dx, dy, "port")
        t = np.array([tau.xy(x, y) for x, y in zip(dx, dy)])
        td = np.array([tau.xy_diff_x(x, y) for x, y in zip(dx, dy)])
        assert (np.abs(t - a) * r).max() <= 1e-8, lo
        assert (np.abs(td - ad) * r * r).max() <= 5e-8, lo


@pytest.mark.gpu
def test_device_tabulated_speeds_and_jacobian(engine_lib, port_lib):
    from sdddst_b200 import capi
    n, m, h = 1024, 1.0, 2e-5
    xyb, _ = workloads.dislocations(n, 13)
    e = capi.Engine(capi.cli_params(n, m, 1e-6, field=capi.FIELD_TABULATED), xyb)
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=1e-6), "port")
    v, tol = e.speeds(xyb)
    v_ref, tol_ref = o.speeds(xyb)
    assert np.abs(v - v_ref).max() <= n * 1e-8, np.abs(v - v_ref).max()
    assert np.array_equal(tol, tol_ref)  # tolerances depend on distances only
    rp, col, val, d = e.jacobian(h, xyb)
    Ap, Ai, Ax, d_ref = o.jacobian(h, xyb)
    J = np.zeros((n, n))
    for i in range(n):
        J[i, col[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]]
    Jr = ref.csc_to_dense(Ap, Ai, Ax, n)
    assert np.array_equal(J != 0, Jr != 0)
    off = ~np.eye(n, dtype=bool)
    assert np.abs(J - Jr).max() <= 1e-6 * np.abs(Jr[off]).max()


@pytest.mark.gpu
def test_device_tabulated_steps(engine_lib):
    """Ten step attempts with the tabulated field stay within 1e-7 of the
    analytic field's trajectory (same accept/reject decisions)."""
    from sdddst_b200 import capi
    n = 512
    xyb, _ = workloads.dislocations(n, 14)
    et = capi.Engine(capi.cli_params(n, 1.0, 1e-6, step_size=1e-6, field=capi.FIELD_TABULATED), xyb)
    ea = capi.Engine(capi.cli_params(n, 1.0, 1e-6, step_size=1e-6), xyb)
    for k in range(10):
        assert et.step() == ea.step(), k
        assert np.abs(et.config(0)[:, 0] - ea.config(0)[:, 0]).max() <= 1e-7, k
