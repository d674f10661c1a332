"""The learned preconditioner correction (SDDDST_SOLVER_GMRES_LEARNED).

* CPU: the shipped weight file has the network's size and round-trips
  through the BF16 packing.
* GPU: the CUDA inference (csrc/learned.cu) against the PyTorch FP32
  definition of the same network (sdddst_b200/learned.py) with the same BF16
  weights, on the same Jacobian and cluster blocks (BF16 operands and FP32
  accumulation in the node products of both, different summation orders:
  a node state or Q h near a BF16 rounding tie can round to neighbouring
  BF16 values, 2^-8 apart, so entries agree within 2e-3 of the largest |C|
  plus 1e-2 relative, the median within 1e-5 of it; C only preconditions
  GMRES, which solves to 1e-13 either way, as the trajectory test checks);
  the learned solver's trajectory against the cluster-preconditioned one
  (both solve to a 1e-13 residual: same decisions, positions within 1e-9).
"""
import numpy as np
import pytest

from sdddst_b200 import learned, workloads


def test_weights_file_shape_and_packing():
    w = learned.load_weights()
    assert w.dtype == np.uint16 and w.size == learned.weight_count()
    torch = pytest.importorskip("torch")
    net = learned.make_net()
    learned.unpack_into(net, w)
    again = learned.pack_bf16(net)
    assert np.array_equal(again, w)
    meta = np.load(learned.WEIGHTS_FILE)["meta"]
    assert "heldout_loss" in str(meta)


def _engine(n, seed, solver):
    from sdddst_b200 import capi
    xyb, _ = workloads.dislocations(n, seed)
    e = capi.Engine(capi.cli_params(n, 2.0, 1e-5, step_size=1e-6, pairsum=capi.PAIRSUM_FP32, solver=solver), xyb)
    if solver == capi.SOLVER_GMRES_LEARNED:
        e.set_preconditioner_weights()
    return e, xyb


@pytest.mark.gpu
def test_learned_inference_matches_torch(engine_lib):
    import torch
    from sdddst_b200 import capi
    n = 2048
    e, xyb = _engine(n, 21, capi.SOLVER_GMRES_LEARNED)
    for _ in range(2):
        e.step()
    h = e.scalars()["step_size"]
    cfg = e.config(0)
    cval = e.learned_correction(h)
    rp, col, val, d = e.jacobian(h, cfg)
    z = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    bz = torch.empty_like(z)
    blk = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    e.precond_apply(h, 1, z.data_ptr(), bz.data_ptr(), blk.data_ptr())
    g = learned.Graph(rp, col, val, d, cfg[:, 0], cfg[:, 1], e.scalars()["cutoff"], blk.cpu().numpy())
    net = learned.make_net()
    learned.unpack_into(net, learned.load_weights())
    with torch.no_grad():
        ce, cd = net(g)
    ref = np.zeros(len(col), dtype=np.float64)
    rows = np.repeat(np.arange(n), np.diff(rp))
    off = col != rows
    ref[off] = (ce.double() * g.scale.double()).numpy()
    ref[~off] = (cd.double() / g.Jii).numpy()[rows[~off]]
    scale = np.abs(ref).max()
    assert scale > 0
    err = np.abs(cval.astype(np.float64) - ref)
    assert np.all(err <= 2e-3 * scale + 1e-2 * np.abs(ref)), (err.max(), scale)
    assert np.median(err) <= 1e-5 * scale, (np.median(err), scale)


@pytest.mark.gpu
def test_learned_solver_matches_cluster_trajectory(engine_lib):
    from sdddst_b200 import capi
    n = 2048
    a, _ = _engine(n, 22, capi.SOLVER_GMRES_LEARNED)
    b, _ = _engine(n, 22, capi.SOLVER_GMRES_CLUSTER)
    for k in range(10):
        assert a.step() == b.step(), k
        assert np.abs(a.config(0)[:, 0] - b.config(0)[:, 0]).max() <= 1e-9, k
    assert a.solver_stats()[0] > 0
    # one inference per attempt: stage II rescales it, stage III's assembly
    # remaps it onto its own pattern
    import ctypes as C
    fn = a.lib.sdddst_internal_learned_counts
    fn.argtypes = [C.c_void_p] + [C.POINTER(C.c_long)] * 3
    fn.restype = C.c_int
    inf, resc, remap = C.c_long(), C.c_long(), C.c_long()
    assert fn(a.h, C.byref(inf), C.byref(resc), C.byref(remap)) == 0
    assert remap.value > 0 and inf.value <= 11, (inf.value, resc.value, remap.value)
