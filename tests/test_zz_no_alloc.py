"""The allocation-free entry point (sdddst_speeds_noalloc).

It serves callers that cannot allocate device memory: their memory is
budgeted by another framework, or a cudaMalloc with its implicit device-wide
synchronisation would stall the work they interleave with.  Its scratch is a
static array inside the library.  This test calls it through the C ABI with
device buffers the test owns, twice in a row (the scratch keeps the previous
call's contents), and checks both results against the regular velocity entry
point with the tolerance of the velocity parity tests.  It runs last so that a
failure here leaves every other test already run, and it passes alone in a
fresh process as well as after the others.
"""
import ctypes as C

import numpy as np
import pytest

from sdddst_b200 import workloads

pytestmark = pytest.mark.gpu


def _tol_ok(v, v_ref):
    return np.all(np.abs(v - v_ref) <= 1e-10 * np.abs(v_ref).max() + 1e-9 * np.abs(v_ref))


def test_speeds_noalloc_matches_regular_entry_point(engine_lib):
    import torch
    from sdddst_b200 import capi
    lib = capi.load()
    for n, seed, tau in ((1000, 31, 0.0), (4096, 32, 0.01)):
        xyb, _ = workloads.dislocations(n, seed)
        eng = capi.Engine(capi.cli_params(n, 1.0, 1e-6, stress_kind=capi.STRESS_CONSTANT, stress_value=tau), xyb)
        v_ref, _ = eng.speeds(xyb)
        eng.close()
        dev = torch.device("cuda", 0)
        x = torch.tensor(xyb[:, 0], dtype=torch.float64, device=dev)
        y = torch.tensor(xyb[:, 1], dtype=torch.float64, device=dev)
        b = torch.tensor(xyb[:, 2], dtype=torch.float64, device=dev)
        for call in range(2):
            v = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            stream = torch.cuda.current_stream().cuda_stream
            rc = lib.sdddst_speeds_noalloc(n, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                           C.c_void_p(b.data_ptr()), float(tau), C.c_void_p(v.data_ptr()),
                                           C.c_void_p(stream))
            assert rc == capi.OK, (n, call, rc)
            torch.cuda.synchronize()
            got = v.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert _tol_ok(got, v_ref), (n, call, np.abs(got - v_ref).max())


def test_speeds_noalloc_rejects_sizes_above_its_scratch(engine_lib):
    import torch
    from sdddst_b200 import capi
    lib = capi.load()
    n = 4097
    buf = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = lib.sdddst_speeds_noalloc(n, p, p, p, 0.0, p, None)
    assert rc == capi.ERR_CAPACITY
