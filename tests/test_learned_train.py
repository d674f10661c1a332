"""Device training of the learned preconditioner correction
(csrc/learned_train.cu) against PyTorch autograd of the same network and
loss (sdddst_b200/learned.py): ||Z - J (B + C) Z||^2 / ||Z||^2 over sign
probes Z on one Jacobian of the N=600 workload (cutoff multiplier 2).

The device gradient uses BF16 operands in its tensor-core weight-gradient
products (the network's node products are BF16 in both), so the bars are a
cosine similarity and a relative norm error, per weight tensor and overall.
"""
import numpy as np
import pytest

from sdddst_b200 import workloads


def _probes(seed, k, n):
    """The device's sign probes: bit 0 of a splitmix-style hash of (seed, p, i)."""
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    p = np.arange(k, dtype=np.uint64)[:, None]
    i = np.arange(n, dtype=np.uint64)[None, :]
    z = (np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * (p + np.uint64(1)) +
         np.uint64(0xBF58476D1CE4E5B9) * (i + np.uint64(1))) & M
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M
    r = z ^ (z >> np.uint64(31))
    return np.where((r & np.uint64(1)) == 1, 1.0, -1.0)


@pytest.mark.gpu
def test_device_gradient_matches_autograd(engine_lib):
    import torch
    from sdddst_b200 import capi, learned
    n, k, seed, h = 600, 4, 7, 3e-5
    xyb, _ = workloads.dislocations(n, 5)
    e = capi.Engine(capi.cli_params(n, 2.0, 1e-5, pairsum=capi.PAIRSUM_FP32, solver=capi.SOLVER_GMRES_LEARNED), xyb)
    w0 = learned.init_weights(3)
    rng = np.random.default_rng(4)
    # output layers away from zero, so that every weight receives a gradient
    off = w0.size - 2 * (learned.H + 1)
    w0[off:] = rng.uniform(-0.2, 0.2, 2 * (learned.H + 1)).astype(np.float32)
    e.learned_train_init(w0)
    loss_b, loss_c, g = e.learned_train_step(h, probes=k, lr=0.0, seed=seed, apply=False, grad=True)

    # the same loss in PyTorch on the device's own J, B and probes
    dev = "cuda"
    cfg = e.config(0)
    rp, col, val, d = e.jacobian(h, cfg)
    Z = torch.tensor(_probes(seed, k, n), dtype=torch.float64, device=dev).contiguous()
    BZ = torch.empty_like(Z)
    blk = torch.empty(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    e.precond_apply(h, k, Z.data_ptr(), BZ.data_ptr(), blk.data_ptr())
    torch.cuda.synchronize()
    graph = learned.Graph(rp, col, val, d, cfg[:, 0], cfg[:, 1], e.scalars()["cutoff"], blk.cpu().numpy(), dev)
    net = learned.make_net().to(dev)
    learned.unpack_into(net, learned.bf16_bits(w0))
    Zt, BZt = Z.T.contiguous(), BZ.T.contiguous()
    R0 = Zt - graph.apply_J(BZt)
    c_e, c_d = net(graph)
    R = R0 - graph.apply_J(graph.apply_C(c_e, c_d, Zt))
    loss = (R ** 2).sum() / (n * k)
    net.zero_grad()
    loss.backward()
    ref_b = float((R0 ** 2).sum()) / (n * k)
    assert abs(loss_b - ref_b) <= 1e-9 * ref_b
    assert abs(loss_c - float(loss)) <= 2e-3 * float(loss)
    # the device's step follows loss / loss_B (the loss with B alone)
    grads = [t.grad.detach().double().cpu().numpy().ravel() / ref_b for t in learned.weight_tensors(net)]
    ref = np.concatenate(grads)
    gd = g.astype(np.float64)
    cos = float(gd @ ref / (np.linalg.norm(gd) * np.linalg.norm(ref)))
    assert cos > 0.995, cos
    assert np.linalg.norm(gd - ref) <= 0.05 * np.linalg.norm(ref)
    at = 0
    for t, r in zip(learned.weight_tensors(net), grads):
        seg = gd[at:at + r.size]
        at += r.size
        if np.linalg.norm(r) > 1e-3 * np.linalg.norm(ref):
            c = float(seg @ r / (np.linalg.norm(seg) * np.linalg.norm(r)))
            assert c > 0.98, (tuple(t.shape), c)


@pytest.mark.gpu
def test_device_training_lowers_the_loss(engine_lib):
    """Adam on the device moves downhill: from the first-order start (zero
    output layers), on one Jacobian of the N=2048 workload at its initial
    step size and one fixed set of probes, a single tiny step lowers the
    loss (Adam's first step moves every weight by the rate, and the loss
    reacts strongly to the output layer), and thirty steps at the trainer's
    rate keep it below the start; the correction the inference computes from
    the refreshed BF16 weights stays finite."""
    from sdddst_b200 import capi, learned
    n = 2048
    xyb, _ = workloads.dislocations(n, 6)
    e = capi.Engine(capi.cli_params(n, 2.0, 1e-5, pairsum=capi.PAIRSUM_FP32, solver=capi.SOLVER_GMRES_LEARNED), xyb)
    e.learned_train_init(learned.init_weights(0))
    h = 1e-6
    _, first = e.learned_train_step(h, probes=8, lr=0.0, seed=999, apply=False)
    e.learned_train_step(h, probes=8, lr=1e-7, seed=999)
    _, one = e.learned_train_step(h, probes=8, lr=0.0, seed=999, apply=False)
    assert one < first, (first, one)
    for _ in range(30):
        e.learned_train_step(h, probes=8, lr=1e-5, seed=999)
    _, last = e.learned_train_step(h, probes=8, lr=0.0, seed=999, apply=False)
    assert last < first, (first, one, last)
    w = e.learned_train_weights()
    corr = e.learned_correction(h)
    assert np.all(np.isfinite(w)) and np.all(np.isfinite(corr))
