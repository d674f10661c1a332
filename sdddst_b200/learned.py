"""Learned correction of the cluster block-Jacobi preconditioner.

The GMRES preconditioner of the learned solver mode is M = B + C:

* B is the cluster block-Jacobi inverse (csrc/precond.cu): strongly coupled
  dislocations are grouped and their diagonal blocks of J inverted exactly;
* C has the sparsity pattern of J (the cutoff-neighbour graph) and its values
  come from a small message-passing network over that graph.

Network (hidden width H = 64, ReLU, weights stored in BF16; the node
products P h, Q h, U [h; a], P_o h, Q_o h take BF16 operands and accumulate
in FP32 (the tensor-core form of csrc/node_gemm_tc.cu), Q h and Q_o h are
kept in BF16, everything else is FP32):

    h_i  = relu(W_in f_i + b_in)                                  node input
    3 x: m_ij = relu(P h_i + b_P + Q h_j + R e_ij)               messages
         a_i  = mean_j m_ij                                       aggregation
         h_i += relu(U [h_i; a_i] + b_U)                          node update
    c_ij = w_o . relu(P_o h_i + b_Po + Q_o h_j + R_o e_ij) + b_o - (1 - s_ij)
    c_ii = w_d . h_i + b_d                                        diagonal output

with s_ij = 1 when i and j share a block of B, and the correction is scaled
by the first-order Neumann term of the matrix, C_ij = c_ij A_ij / (J_ii J_jj),
C_ii = c_ii / J_ii, where J = I + A, A = diag((1 + d)/2) h G.  With the
output layers at zero the network reproduces the analytic first-order
block-Neumann correction (c_ij = -1 across blocks, 0 inside them); training
learns the residual over it.  The message function is linear in [h_i; h_j; e_ij]
before its activation, so its weights split into per-node projections
(P h, Q h: N x 64 x 64 products) and a per-edge sum: no edge-sized matrix
product exists.

Features (scale-free; t(v) = sign(v) log(1 + |v|)):
    node f_i = [t(A_ii), t(sum_j |A_ij|), t(sum_j |A_ji|), deg_i / 627]
    edge e_ij = [t(A_ij), t(A_ji), dx / 7c, dy / 7c, same_block(i, j)]
with dx, dy the minimum-image separation x_j - x_i, y_j - y_i, c the cutoff
and same_block 1 when i and j share a block of B.

Training minimises the probe estimate of ||I - J (B + C)||_F^2 over Jacobians
produced by runs of the method (learned_train.py).  This module holds the
PyTorch definition (training, and the reference of the CUDA inference in
csrc/learned.cu), the features and the flat BF16 weight layout loaded through
sdddst_set_preconditioner_weights.
"""
from __future__ import annotations

import os

import numpy as np

H = 64
NODE_F = 4
EDGE_F = 5
LAYERS = 3
DEG_SCALE = 627.0
POS_SCALE = 7.0
WEIGHTS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "learned_weights.npz")


def _torch():
    import torch
    return torch


def tlog(v):
    torch = _torch()
    return torch.sign(v) * torch.log1p(v.abs())


class Graph:
    """CSR of J (diagonal in each row's first slot, as exported) with the
    per-edge and per-node quantities the network and the loss use."""

    def __init__(self, rowptr, col, val, dvec, x, y, cutoff, block, device="cpu"):
        torch = _torch()
        t = lambda a, dt: torch.as_tensor(np.asarray(a), dtype=dt, device=device)
        rowptr = t(rowptr, torch.int64)
        col = t(col, torch.int64)
        val = t(val, torch.float64)
        dvec = t(dvec, torch.float64)
        x, y = t(x, torch.float64), t(y, torch.float64)
        block = t(block, torch.int64)
        n = rowptr.numel() - 1
        counts = rowptr[1:] - rowptr[:-1]
        row = torch.repeat_interleave(torch.arange(n, device=device), counts)
        diag = col == row
        self.n = n
        self.Aii = torch.zeros(n, dtype=torch.float64, device=device).index_add_(0, row[diag], val[diag] - 1.0)
        off = ~diag
        self.r, self.c = row[off], col[off]
        self.Aij = val[off]
        self.Aji = self.Aij * (1.0 + dvec[self.c]) / (1.0 + dvec[self.r])
        self.Jii = 1.0 + self.Aii
        deg = torch.zeros(n, dtype=torch.float64, device=device).index_add_(0, self.r, torch.ones_like(self.Aij))
        self.deg = deg
        rs = torch.zeros(n, dtype=torch.float64, device=device).index_add_(0, self.r, self.Aij.abs())
        cs = torch.zeros(n, dtype=torch.float64, device=device).index_add_(0, self.r, self.Aji.abs())
        self.node_f = torch.stack([tlog(self.Aii), tlog(rs), tlog(cs), deg / DEG_SCALE], 1).float()
        dx = x[self.c] - x[self.r]
        dy = y[self.c] - y[self.r]
        dx = dx - torch.round(dx)
        dy = dy - torch.round(dy)
        same = (block[self.c] == block[self.r]).double()
        self.edge_f = torch.stack([tlog(self.Aij), tlog(self.Aji), dx / (POS_SCALE * cutoff),
                                   dy / (POS_SCALE * cutoff), same], 1).float()
        self.scale = (self.Aij / (self.Jii[self.r] * self.Jii[self.c])).float()

    def apply_J(self, Y):
        """J Y for Y of shape (n, k)."""
        out = Y * (1.0 + self.Aii)[:, None].to(Y.dtype)
        return out.index_add(0, self.r, self.Aij[:, None].to(Y.dtype) * Y[self.c])

    def apply_C(self, c_edge, c_diag, Y):
        """C Y with C_ij = c_ij A_ij / (J_ii J_jj), C_ii = c_ii / J_ii."""
        ce = (c_edge * self.scale).to(Y.dtype)
        out = Y * (c_diag.to(Y.dtype) / self.Jii.to(Y.dtype))[:, None]
        return out.index_add(0, self.r, ce[:, None] * Y[self.c])


def make_net():
    torch = _torch()
    nn = torch.nn

    class Net(nn.Module):
        def __init__(self):
            super().__init__()
            self.inp = nn.Linear(NODE_F, H)
            self.P = nn.ModuleList([nn.Linear(H, H) for _ in range(LAYERS)])
            self.Q = nn.ModuleList([nn.Linear(H, H, bias=False) for _ in range(LAYERS)])
            self.R = nn.ModuleList([nn.Linear(EDGE_F, H, bias=False) for _ in range(LAYERS)])
            self.U = nn.ModuleList([nn.Linear(2 * H, H) for _ in range(LAYERS)])
            self.Po = nn.Linear(H, H)
            self.Qo = nn.Linear(H, H, bias=False)
            self.Ro = nn.Linear(EDGE_F, H, bias=False)
            self.wo = nn.Linear(H, 1)
            self.wd = nn.Linear(H, 1)

        def forward(self, g):
            relu = torch.relu
            # the node products take BF16 operands (node states rounded to
            # BF16, BF16 weights) and accumulate in FP32, as on the tensor
            # cores; Q h is kept in BF16 for the per-edge gather
            bf = lambda t: t.to(torch.bfloat16).float()
            h = relu(self.inp(g.node_f))
            deg = g.deg.float().clamp(min=1.0)[:, None]
            for l in range(LAYERS):
                ph, qh = self.P[l](bf(h)), bf(self.Q[l](bf(h)))
                m = relu(ph[g.r] + qh[g.c] + self.R[l](g.edge_f))
                a = torch.zeros_like(h).index_add_(0, g.r, m) / deg
                h = h + relu(self.U[l](torch.cat([bf(h), bf(a)], 1)))
            po, qo = self.Po(bf(h)), bf(self.Qo(bf(h)))
            c_edge = self.wo(relu(po[g.r] + qo[g.c] + self.Ro(g.edge_f))).squeeze(1) - (1.0 - g.edge_f[:, 4])
            c_diag = self.wd(h).squeeze(1)
            return c_edge, c_diag

    return Net()


def weight_tensors(net):
    """Tensors in the flat order of the C ABI's weight array."""
    out = [net.inp.weight, net.inp.bias]
    for l in range(LAYERS):
        out += [net.P[l].weight, net.P[l].bias, net.Q[l].weight, net.R[l].weight, net.U[l].weight, net.U[l].bias]
    out += [net.Po.weight, net.Po.bias, net.Qo.weight, net.Ro.weight, net.wo.weight, net.wo.bias,
            net.wd.weight, net.wd.bias]
    return out


def weight_count():
    per_layer = H * H + H + H * H + H * EDGE_F + H * 2 * H + H
    return H * NODE_F + H + LAYERS * per_layer + H * H + H + H * H + H * EDGE_F + H + 1 + H + 1


def init_weights(seed: int = 0) -> np.ndarray:
    """Flat FP32 starting weights for the device trainer: every layer as
    PyTorch's nn.Linear initialises it (weights and biases uniform in
    +-1/sqrt(fan_in)), the output layers (w_o, b_o, w_d, b_d) at zero, so the
    correction starts as the analytic first-order term."""
    rng = np.random.default_rng(seed)
    parts = []

    def lin(out_f, in_f, bias=True):
        b = 1.0 / np.sqrt(in_f)
        parts.append(rng.uniform(-b, b, out_f * in_f))
        if bias:
            parts.append(rng.uniform(-b, b, out_f))

    lin(H, NODE_F)
    for _ in range(LAYERS):
        lin(H, H)              # P, b_P
        lin(H, H, bias=False)  # Q
        lin(H, EDGE_F, False)  # R
        lin(H, 2 * H)          # U, b_U
    lin(H, H)                  # P_o, b_Po
    lin(H, H, bias=False)      # Q_o
    lin(H, EDGE_F, False)      # R_o
    parts.append(np.zeros(H + 1))  # w_o, b_o
    parts.append(np.zeros(H + 1))  # w_d, b_d
    w = np.concatenate(parts).astype(np.float32)
    assert w.size == weight_count()
    return w


def bf16_bits(w: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 bit patterns (uint16), round to nearest even."""
    bits = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).astype(np.uint16)


def pack_bf16(net) -> np.ndarray:
    """Flat BF16 bit patterns (uint16), round to nearest even."""
    flat = np.concatenate([t.detach().float().cpu().numpy().ravel() for t in weight_tensors(net)])
    assert flat.size == weight_count()
    bits = flat.astype(np.float32).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) >> 16
    return rounded.astype(np.uint16)


def unpack_into(net, bf16: np.ndarray):
    """Loads flat BF16 weights into a PyTorch network (FP32 parameters)."""
    torch = _torch()
    f = (bf16.astype(np.uint32) << 16).view(np.float32)
    off = 0
    with torch.no_grad():
        for t in weight_tensors(net):
            k = t.numel()
            t.copy_(torch.from_numpy(f[off:off + k].copy()).view_as(t))
            off += k
    assert off == f.size


def load_weights(path: str = WEIGHTS_FILE) -> np.ndarray:
    return np.load(path)["bf16"]
