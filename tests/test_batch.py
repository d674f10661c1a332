"""Batched stepping of independent systems of uneven size (one launch per
phase for all systems) against independent oracle runs of each system."""
import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads

pytestmark = pytest.mark.gpu


def test_batch_matches_independent_systems(engine_lib, port_lib):
    from sdddst_b200 import capi
    sizes = [64, 97, 150, 203, 256, 300]
    systems = [workloads.dislocations(n, 500 + k)[0] for k, n in enumerate(sizes)]
    prm = capi.default_params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6)
    bt = capi.Batch(prm, systems)
    oracles = [ref.Sim(s, None, ref.params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6), "port")
               for s in systems]
    assert bt.info()["tile"] in (32, 64, 128)
    for step in range(12):
        acc = bt.step()
        acc_ref = np.array([o.step() for o in oracles])
        assert np.array_equal(acc, acc_ref), step
        xs = bt.positions(0)
        sc = bt.scalars()
        for k, o in enumerate(oracles):
            assert np.abs(xs[k] - o.config(0)[:, 0]).max() <= 1e-9, (step, k)
            s = o.scalars()
            assert np.isclose(sc[k, 1], s["step_size"], rtol=1e-6), (step, k)
            assert np.isclose(sc[k, 0], s["sim_time"], rtol=1e-6, atol=0)
            assert sc[k, 2] == s["successful_steps"] and sc[k, 3] == s["failed_steps"]
            assert np.isclose(sc[k, 4], s["energy"], rtol=1e-8)
    bt.close()


def test_batch_mixed_precision_runs(engine_lib):
    from sdddst_b200 import capi
    sizes = workloads.batch_sizes(40, 3)
    systems = [workloads.dislocations(int(n), 900 + k)[0] for k, n in enumerate(sizes)]
    p64 = capi.default_params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6)
    p32 = capi.default_params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6, pairsum=capi.PAIRSUM_FP32)
    a, b = capi.Batch(p64, systems), capi.Batch(p32, systems)
    for _ in range(3):
        acc_a, acc_b = a.step(), b.step()
        same = acc_a == acc_b
        for k in np.nonzero(same)[0]:
            assert np.abs(a.positions(0)[k] - b.positions(0)[k]).max() < 1e-8
