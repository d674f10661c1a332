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


def test_batch_workload_systems_match_oracle(engine_lib, port_lib):
    """Eight systems of the batched workload itself (sizes drawn from
    U[64, 2048] with seed 3, each system's own seed; cutoff multiplier 0.5,
    precision 1e-6): per-system decisions, positions, step sizes, times,
    counters and energies against independent oracle runs over 6 attempts,
    with the systems accepting and rejecting unevenly."""
    from concurrent.futures import ThreadPoolExecutor
    from sdddst_b200 import capi
    sizes = workloads.batch_sizes(workloads.BATCH_COUNT, workloads.BATCH_SEED)[:8]
    systems = [workloads.dislocations(int(n), workloads.BATCH_SEED * 100003 + k)[0] for k, n in enumerate(sizes)]
    prm = capi.default_params(cutoff_multiplier=workloads.BATCH_M, prec=1e-6, step_size=1e-6)
    bt = capi.Batch(prm, systems)
    oracles = [ref.Sim(s, None, ref.params(cutoff_multiplier=workloads.BATCH_M, prec=1e-6, step_size=1e-6), "port")
               for s in systems]
    uneven = False
    with ThreadPoolExecutor(max_workers=8) as pool:  # the oracle releases the GIL inside its C calls
        for step in range(6):
            acc = bt.step()
            acc_ref = np.array(list(pool.map(lambda o: o.step(), oracles)))
            assert np.array_equal(acc, acc_ref), step
            uneven |= bool(acc.any() and not acc.all())
            xs = bt.positions(0)
            sc = bt.scalars()
            for k, o in enumerate(oracles):
                assert np.abs(xs[k] - o.config(0)[:, 0]).max() <= 1e-9, (step, k)
                s = o.scalars()
                assert np.isclose(sc[k, 1], s["step_size"], rtol=1e-6), (step, k)
                assert np.isclose(sc[k, 0], s["sim_time"], rtol=1e-6, atol=0)
                assert sc[k, 2] == s["successful_steps"] and sc[k, 3] == s["failed_steps"]
                assert np.isclose(sc[k, 4], s["energy"], rtol=1e-8)
    assert uneven, "every attempt was accepted or rejected by all systems together"
    # after the host-driven first step, every step replays the captured graph
    assert bt.stats() == {"graph": 1, "redone": 0}, bt.stats()
    bt.close()
