// Learned correction C of the cluster block-Jacobi preconditioner B: the
// GMRES preconditioner of SDDDST_SOLVER_GMRES_LEARNED is M = B + C, C on the
// sparsity pattern of J, its values from a message-passing network over the
// cutoff-neighbour graph (hidden width 64, three rounds, ReLU).  Weights are
// held in BF16.  The node products (P h, Q h, U [h; a], P_o h, Q_o h) run on
// the tensor cores (node_gemm_tc.cu: BF16 node states and weights, FP32
// accumulation in tensor memory; Q h kept in BF16 for the edge pass's
// gather); the per-edge sums and the small input and output layers are FP32
// on the CUDA cores.
//
//   h_i  = relu(W_in f_i + b_in)
//   3 x: m_ij = relu(P h_i + b_P + Q h_j + R e_ij), a_i = mean_j m_ij,
//        h_i += relu(U [h_i; a_i] + b_U)
//   c_ij = w_o . relu(P_o h_i + b_Po + Q_o h_j + R_o e_ij) + b_o - (1 - s_ij),  c_ii = w_d . h_i + b_d
//   C_ij = c_ij A_ij / (J_ii J_jj),  C_ii = c_ii / J_ii,   J = I + A, A = diag((1+d)/2) h G
// (s_ij = 1 when i and j share a cluster block; with zero output layers C is
// the analytic first-order block-Neumann correction, which
// SDDDST_SOLVER_GMRES_NEUMANN uses without the network)
//
// Features (t(v) = sign(v) log(1 + |v|)): node [t(A_ii), t(sum_j |A_ij|),
// t(sum_j |A_ji|), deg / 627]; edge [t(A_ij), t(A_ji), dx / 7c, dy / 7c,
// same cluster block].  The message function is linear in [h_i; h_j; e_ij]
// before its activation, so it splits into per-node projections (P h, Q h:
// N x 64 x 64 products, on the tensor cores) and a per-edge sum over the CSR
// rows (one warp per row, two channels per lane); no edge-sized matrix
// product exists.  The flat weight order and the features follow
// sdddst_b200/learned.py, the PyTorch definition the network was trained in.
#include <cuda_bf16.h>

#include <vector>

#include "common.cuh"
#include "engine.h"
#include "learned_net.cuh"

#include <utility>

namespace sd {

using namespace ln;

__global__ void scan_kernel(const int *__restrict__ in, int m, int *__restrict__ out);

namespace {

// analytic first-order block-Neumann correction: C_ij = -A_ij / (J_ii J_jj)
// across cluster blocks, 0 inside them and on the diagonal
template <typename VT>
__global__ void first_order_kernel(int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                                   const VT *__restrict__ val, const double *__restrict__ dvec,
                                   const double *__restrict__ jii, const int *__restrict__ blk, double theta2,
                                   float *__restrict__ cval)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double di = (1.0 + dvec[i]) * 0.5 * h, ji = jii[i];
    const int bi = blk[i];
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) {
        const int j = col[q];
        float v = 0.0f;
        if (j != i && blk[j] != bi) {
            const double aij = di * (double)val[q], jj = jii[j];
            if (fabs(aij) >= theta2 * sqrt(fabs(ji * jj))) v = (float)(-aij / (ji * jj));
        }
        cval[q] = v;
    }
}

// compaction of the analytic correction's nonzero off-diagonals into its own
// CSR (column positions in the cell-sorted order), one warp per row
__global__ void c_count_kernel(int n, const int *__restrict__ rowptr, const float *__restrict__ cval,
                               int *__restrict__ cnt)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    int c = 0;
    for (int q = rowptr[i] + 1 + lane; q < rowptr[i + 1]; q += 32) c += cval[q] != 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[i] = c;
}

__global__ void c_fill_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col_s,
                              const float *__restrict__ cval, const int *__restrict__ crow, int *__restrict__ ccol,
                              float *__restrict__ cv)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    int at = crow[i];
    for (int q0 = rowptr[i] + 1; q0 < rowptr[i + 1]; q0 += 32) {
        const int q = q0 + lane;
        const bool keep = q < rowptr[i + 1] && cval[q] != 0.0f;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int o = at + __popc(m & ((1u << lane) - 1u));
            ccol[o] = col_s[q];
            cv[o] = cval[q];
        }
        at += __popc(m);
    }
}

// z += C v over the compact correction (v gathered in the cell-sorted order)
__global__ void c_apply_kernel(int n, const int *__restrict__ crow, const int *__restrict__ ccol,
                               const float *__restrict__ cv, const double *__restrict__ vs, double *__restrict__ z)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    double acc = 0.0;
    for (int q = crow[i] + lane; q < crow[i + 1]; q += 32) acc += (double)cv[q] * vs[ccol[q]];
    acc = warp_sum(acc);
    if (lane == 0 && crow[i + 1] > crow[i]) z[i] += acc;
}

// C for J(h') from the network outputs of another step size on the same
// assembly: C_ij = (c_ij - (1 - s_ij)) A_ij / (J_ii J_jj), C_ii = c_ii / J_ii
// with A, J and the cluster blocks s of h' (one warp per row).  The network
// runs once per assembly; stage II's J(h/2) reuses stage I's outputs.
template <typename VT>
__global__ void rescale_kernel(int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                               const VT *__restrict__ val, const double *__restrict__ gdiag,
                               const double *__restrict__ dvec, const int *__restrict__ blk,
                               const float *__restrict__ craw, const float *__restrict__ crawd,
                               float *__restrict__ cval)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double di = (1.0 + dvec[i]) * 0.5 * h;
    const double ji = 1.0 + di * gdiag[i];
    const int bi = blk[i];
    const int s = rowptr[i], e = rowptr[i + 1];
    for (int q = s + lane; q < e; q += 32) {
        const int j = col[q];
        if (j == i) {
            cval[q] = (float)(crawd[i] / ji);
            continue;
        }
        const double aij = di * (double)val[q];
        const double jj = 1.0 + (1.0 + dvec[j]) * 0.5 * h * gdiag[j];
        const float sc = (float)(aij / (ji * jj));
        const float e4 = blk[j] == bi ? 1.0f : 0.0f;
        cval[q] = (craw[q] - (1.0f - e4)) * sc;
    }
}

// The network's raw outputs of the previous assembly's pattern (rp0, col0)
// carried onto the current one, one warp per row: a row whose columns are
// unchanged copies them; otherwise every entry looks for its column in the
// old row, first within eight slots of its own offset (a few entries came or
// went), then over the whole row, and takes 0 where the column is new (the
// network's part of c_ij, leaving the analytic first-order value).
__global__ void remap_raw_kernel(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                 const int *__restrict__ rp0, const int *__restrict__ col0,
                                 const float *__restrict__ raw0, float *__restrict__ raw)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int s = rp[i], e = rp[i + 1], s0 = rp0[i], e0 = rp0[i + 1];
    const int len = e - s, len0 = e0 - s0;
    bool same = len == len0;
    if (same)
        for (int k = lane; k < len; k += 32) same = same && col[s + k] == col0[s0 + k];
    same = __all_sync(0xffffffffu, same);
    if (same) {
        for (int k = lane; k < len; k += 32) raw[s + k] = raw0[s0 + k];
        return;
    }
    for (int k = 1 + lane; k < len; k += 32) { // slot 0 is the diagonal
        const int j = col[s + k];
        int at = -1;
        for (int d = 0; d <= 8 && at < 0; ++d) {
            if (k + d < len0 && col0[s0 + k + d] == j) at = k + d;
            else if (d > 0 && k - d >= 1 && k - d < len0 && col0[s0 + k - d] == j) at = k - d;
        }
        for (int k0 = 1; k0 < len0 && at < 0; ++k0)
            if (col0[s0 + k0] == j) at = k0;
        raw[s + k] = at >= 0 ? raw0[s0 + at] : 0.0f;
    }
    if (lane == 0) raw[s] = raw0[s0];
}

// z += C v, one warp per row
__global__ void apply_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                             const float *__restrict__ cval, const double *__restrict__ v, double *__restrict__ z)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    double acc = 0.0;
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) acc += (double)cval[q] * v[col[q]];
    acc = warp_sum(acc);
    if (lane == 0) z[i] += acc;
}

// z += C v with the off-diagonal gathers from vs, v in the cell-sorted order
__global__ void apply_sorted_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col_s,
                                    const float *__restrict__ cval, const double *__restrict__ v,
                                    const double *__restrict__ vs, double *__restrict__ z)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int s = rowptr[i], e = rowptr[i + 1];
    double acc = lane == 0 ? (double)cval[s] * v[i] : 0.0; // diagonal slot
    for (int q = s + 1 + lane; q < e; q += 32) acc += (double)cval[q] * vs[col_s[q]];
    acc = warp_sum(acc);
    if (lane == 0) z[i] += acc;
}

__global__ void gather_sorted_v_kernel(int n, const int *__restrict__ sorted, const double *__restrict__ v,
                                       double *__restrict__ vs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) vs[k] = v[sorted[k]];
}

} // namespace

int learned_ensure(Engine &e)
{
    if (e.learned) return 0;
    Learned *L = new Learned();
    e.learned = L;
    const size_t nh = (size_t)e.n * kH;
    const bool ok = cudaMalloc(&L->d_w, sizeof(__nv_bfloat16) * offsets().total) == cudaSuccess &&
                    cudaMalloc(&L->d_nf, sizeof(float) * 4 * e.n) == cudaSuccess &&
                    cudaMalloc(&L->d_h, sizeof(float) * nh) == cudaSuccess &&
                    cudaMalloc(&L->d_ph, sizeof(float) * nh) == cudaSuccess &&
                    cudaMalloc(&L->d_qh, sizeof(__nv_bfloat16) * nh) == cudaSuccess &&
                    cudaMalloc(&L->d_err, sizeof(int)) == cudaSuccess &&
                    cudaMallocHost(&L->h_err, sizeof(int)) == cudaSuccess &&
                    cudaMemset(L->d_err, 0, sizeof(int)) == cudaSuccess &&
                    cudaMalloc(&L->d_agg, sizeof(float) * nh) == cudaSuccess &&
                    cudaMalloc(&L->d_crawd, sizeof(float) * e.n) == cudaSuccess &&
                    cudaMalloc(&L->d_jii, sizeof(double) * e.n) == cudaSuccess;
    if (!ok) {
        e.err = "learned preconditioner: out of device memory";
        return SDDDST_ERR_NOMEM;
    }
    return 0;
}

int learned_set_weights(Engine &e, const unsigned short *bf16, long count)
{
    const WeightOffsets o = offsets();
    if (count != o.total) {
        e.err = "learned preconditioner: expected " + std::to_string(o.total) + " weights, got " +
                std::to_string(count);
        return SDDDST_ERR_INVALID;
    }
    if (int rc = learned_ensure(e)) return rc;
    Learned &L = *LN(e);
    L.off = o;
    cudaMemcpyAsync(L.d_w, bf16, sizeof(unsigned short) * o.total, cudaMemcpyHostToDevice, e.st);
    L.has_weights = true;
    L.raw_valid = L.prev_valid = false; // outputs of other weights are not reused
    return e.sync_check("learned weights");
}

// C for the assembled J(h); the cluster preconditioner must be built (its
// block indices are an edge feature).  analytic: the first-order
// block-Neumann correction without the network.
static void keep_pattern(Engine &e, Learned &L);

int learned_build(Engine &e, double h, const double *dvec, const double *x, bool analytic)
{
    if (!analytic && !(e.learned && LN(e)->has_weights)) {
        e.err = "learned preconditioner: no weights loaded (sdddst_set_preconditioner_weights)";
        return SDDDST_ERR_INVALID;
    }
    if (int rc = learned_ensure(e)) return rc;
    Learned &L = *LN(e);
    if (e.nnz > L.cval_cap) {
        if (L.d_cval) cudaFree(L.d_cval);
        if (L.d_craw) cudaFree(L.d_craw);
        if (L.d_craw0) cudaFree(L.d_craw0);
        if (L.d_col0) cudaFree(L.d_col0);
        L.d_cval = nullptr;
        L.d_craw = nullptr;
        L.d_craw0 = nullptr; // the remap buffers follow cval_cap (they swap with d_craw)
        L.d_col0 = nullptr;
        L.col0_cap = 0;
        L.prev_valid = false;
        L.cval_cap = 0;
        const long cap = e.nnz + e.nnz / 8;
        if (cudaMalloc(&L.d_cval, sizeof(float) * cap) != cudaSuccess ||
            cudaMalloc(&L.d_craw, sizeof(float) * cap) != cudaSuccess) {
            e.err = "learned preconditioner: out of device memory";
            return SDDDST_ERR_NOMEM;
        }
        L.cval_cap = cap;
    }
    const WeightOffsets &o = L.off;
    const int n = e.n;
    cudaStream_t st = e.st;
    const unsigned wrows = (unsigned)((n + 7) / 8); // 8 warps per CTA, one row each
    if (e.valf)
        feat_kernel<float><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_valf, e.d_gdiag, dvec, L.d_nf,
                                                  L.d_jii);
    else
        feat_kernel<double><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_val, e.d_gdiag, dvec, L.d_nf,
                                                   L.d_jii);
    if (analytic) {
        const double th2 = e.prm.neumann_theta > 0 ? e.prm.neumann_theta : 0.0;
        if (e.valf)
            first_order_kernel<float><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_valf, dvec, L.d_jii,
                                                             e.pc.blk_of, th2, L.d_cval);
        else
            first_order_kernel<double><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_val, dvec, L.d_jii,
                                                              e.pc.blk_of, th2, L.d_cval);
        e.launches += 2;
        L.compact = false;
        if (th2 > 0.0 && e.col_s_valid && !e.d_hrow) {
            // thresholded: keep the surviving entries in their own CSR
            if (!L.d_crow && (cudaMalloc(&L.d_crow, sizeof(int) * (n + 1)) != cudaSuccess ||
                              cudaMalloc(&L.d_ccnt, sizeof(int) * (n + 1)) != cudaSuccess)) {
                e.err = "learned preconditioner: out of device memory";
                return SDDDST_ERR_NOMEM;
            }
            if (L.cval_cap > L.ccap) {
                if (L.d_ccol) cudaFree(L.d_ccol);
                if (L.d_cv) cudaFree(L.d_cv);
                L.d_ccol = nullptr;
                L.d_cv = nullptr;
                L.ccap = 0;
                if (cudaMalloc(&L.d_ccol, sizeof(int) * L.cval_cap) != cudaSuccess ||
                    cudaMalloc(&L.d_cv, sizeof(float) * L.cval_cap) != cudaSuccess) {
                    e.err = "learned preconditioner: out of device memory";
                    return SDDDST_ERR_NOMEM;
                }
                L.ccap = L.cval_cap;
            }
            c_count_kernel<<<wrows, 256, 0, st>>>(n, e.d_rowptr, L.d_cval, L.d_ccnt);
            scan_kernel<<<1, 1024, 0, st>>>(L.d_ccnt, n, L.d_crow);
            c_fill_kernel<<<wrows, 256, 0, st>>>(n, e.d_rowptr, e.d_col_s, L.d_cval, L.d_crow, L.d_ccol, L.d_cv);
            e.launches += 3;
            L.compact = true;
        }
        L.builds++;
        return 0;
    }
    if (*L.h_err) { // the previous build's tensor-core wait ran out
        e.err = "learned preconditioner: a tensor-core product did not complete";
        return SDDDST_ERR_CUDA;
    }
    node_in_kernel<<<(unsigned)(((long)n * kH + 255) / 256), 256, 0, st>>>(n, L.d_nf, L.d_w, o.in_w, o.in_b, L.d_h);
    for (int l = 0; l < kLayers; ++l) {
        launch_node_proj_tc(n, L.d_h, L.d_w, o.P[l], o.Pb[l], o.Q[l], L.d_ph, L.d_qh, L.d_err, st);
        if (e.valf)
            edge_kernel<float, false><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_valf, dvec, L.d_jii, x,
                                                             e.d_y, e.pc.blk_of, e.cutoff, L.d_ph, L.d_qh, L.d_w,
                                                             o.R[l], 0, 0, L.d_agg, nullptr, nullptr);
        else
            edge_kernel<double, false><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_val, dvec, L.d_jii, x,
                                                              e.d_y, e.pc.blk_of, e.cutoff, L.d_ph, L.d_qh, L.d_w,
                                                              o.R[l], 0, 0, L.d_agg, nullptr, nullptr);
        launch_node_update_tc(n, L.d_h, L.d_agg, L.d_w, o.U[l], o.Ub[l], L.d_err, st);
    }
    launch_node_proj_tc(n, L.d_h, L.d_w, o.Po, o.Pob, o.Qo, L.d_ph, L.d_qh, L.d_err, st);
    if (e.valf)
        edge_kernel<float, true><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_valf, dvec, L.d_jii, x, e.d_y,
                                                        e.pc.blk_of, e.cutoff, L.d_ph, L.d_qh, L.d_w, o.Ro, o.wo,
                                                        o.wob, nullptr, L.d_cval, L.d_craw);
    else
        edge_kernel<double, true><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, e.d_val, dvec, L.d_jii, x,
                                                         e.d_y, e.pc.blk_of, e.cutoff, L.d_ph, L.d_qh, L.d_w, o.Ro,
                                                         o.wo, o.wob, nullptr, L.d_cval, L.d_craw);
    diag_out_kernel<<<wrows, 256, 0, st>>>(n, L.d_h, L.d_w, o.wd, o.wdb, L.d_jii, e.d_rowptr, L.d_cval, L.d_crawd);
    cudaMemcpyAsync(L.h_err, L.d_err, sizeof(int), cudaMemcpyDeviceToHost, st); // read at the next build
    e.launches += 4 + 3 * kLayers + 2;
    L.builds++;
    L.raw_valid = true;
    keep_pattern(e, L);
    L.remaps = 0;
    return 0;
}

// The current pattern becomes the one the raw outputs belong to.
static void keep_pattern(Engine &e, Learned &L)
{
    L.prev_valid = false;
    if (e.nnz <= 0 || e.d_hrow || e.nnz > L.cval_cap) return;
    if (L.col0_cap != L.cval_cap) { // d_craw0 swaps with d_craw: the same capacity
        if (L.d_col0) cudaFree(L.d_col0);
        if (L.d_craw0) cudaFree(L.d_craw0);
        L.d_col0 = nullptr;
        L.d_craw0 = nullptr;
        L.col0_cap = 0;
        if (cudaMalloc(&L.d_col0, sizeof(int) * L.cval_cap) != cudaSuccess ||
            cudaMalloc(&L.d_craw0, sizeof(float) * L.cval_cap) != cudaSuccess)
            return; // no remapping: the next assembly runs the network
        L.col0_cap = L.cval_cap;
    }
    if (!L.d_rp0 && cudaMalloc(&L.d_rp0, sizeof(int) * (e.n + 1)) != cudaSuccess) return;
    cudaMemcpyAsync(L.d_rp0, e.d_rowptr, sizeof(int) * (e.n + 1), cudaMemcpyDeviceToDevice, e.st);
    cudaMemcpyAsync(L.d_col0, e.d_col, sizeof(int) * e.nnz, cudaMemcpyDeviceToDevice, e.st);
    L.prev_valid = true;
}

// C of the network for J(h) on a new assembly from the outputs of the
// inference on the previous one (one remap per inference: the stage III
// assembly of an attempt reuses the inference of its stage I, whose
// positions differ by a half step); false when that is not possible: run
// learned_build.
bool learned_remap(Engine &e, double h, const double *dvec)
{
    Learned *Lp = LN(e);
    if (!Lp || !Lp->has_weights || !Lp->prev_valid || Lp->remaps >= 1 || e.d_hrow) return false;
    Learned &L = *Lp;
    if (e.nnz <= 0 || e.nnz > L.cval_cap || L.col0_cap != L.cval_cap) return false;
    const unsigned wrows = (unsigned)((e.n + 7) / 8);
    remap_raw_kernel<<<wrows, 256, 0, e.st>>>(e.n, e.d_rowptr, e.d_col, L.d_rp0, L.d_col0, L.d_craw, L.d_craw0);
    std::swap(L.d_craw, L.d_craw0); // both hold cval_cap floats
    e.launches++;
    L.raw_valid = true;
    L.remaps++;
    L.remap_count++;
    keep_pattern(e, L);
    return learned_rescale(e, h, dvec);
}

// C of the network for J(h) from the outputs of the last inference on the
// same assembly (false when there is none: run learned_build)
bool learned_rescale(Engine &e, double h, const double *dvec)
{
    Learned *Lp = LN(e);
    if (!Lp || !Lp->raw_valid || !Lp->has_weights) return false;
    const unsigned wrows = (unsigned)((e.n + 7) / 8);
    if (e.valf)
        rescale_kernel<float><<<wrows, 256, 0, e.st>>>(e.n, h, e.d_rowptr, e.d_col, e.d_valf, e.d_gdiag, dvec,
                                                       e.pc.blk_of, Lp->d_craw, Lp->d_crawd, Lp->d_cval);
    else
        rescale_kernel<double><<<wrows, 256, 0, e.st>>>(e.n, h, e.d_rowptr, e.d_col, e.d_val, e.d_gdiag, dvec,
                                                        e.pc.blk_of, Lp->d_craw, Lp->d_crawd, Lp->d_cval);
    e.launches++;
    Lp->rescales++;
    return true;
}

void learned_counts(Engine &e, long *inferences, long *rescales, long *remaps)
{
    const Learned *L = LN(e);
    *inferences = L ? L->builds : 0;
    *rescales = L ? L->rescales : 0;
    *remaps = L ? L->remap_count : 0;
}

// a new assembly: the network's outputs no longer match the pattern
void learned_invalidate(Engine &e)
{
    if (Learned *Lp = LN(e)) Lp->raw_valid = false;
}

void learned_apply_add(Engine &e, const double *v, double *z)
{
    Learned &L = *LN(e);
    if (L.compact) {
        gather_sorted_v_kernel<<<(unsigned)((e.n + 255) / 256), 256, 0, e.st>>>(e.n, e.spmv_sorted, v, e.d_vsort);
        c_apply_kernel<<<(unsigned)((e.n + 7) / 8), 256, 0, e.st>>>(e.n, L.d_crow, L.d_ccol, L.d_cv, e.d_vsort, z);
        e.launches += 2;
        return;
    }
    if (e.col_s_valid && !e.d_hrow) { // contiguous gathers (the SpMV's staging buffer, free here)
        gather_sorted_v_kernel<<<(unsigned)((e.n + 255) / 256), 256, 0, e.st>>>(e.n, e.spmv_sorted, v, e.d_vsort);
        apply_sorted_kernel<<<(unsigned)((e.n + 7) / 8), 256, 0, e.st>>>(e.n, e.d_rowptr, e.d_col_s, L.d_cval, v,
                                                                         e.d_vsort, z);
        e.launches += 2;
        return;
    }
    apply_kernel<<<(unsigned)((e.n + 7) / 8), 256, 0, e.st>>>(e.n, e.d_rowptr, e.d_col, L.d_cval, v, z);
    e.launches++;
}

int learned_export(Engine &e, float *host, long cap)
{
    Learned *Lp = LN(e);
    if (!Lp || !Lp->d_cval) return SDDDST_ERR_INVALID;
    if (cap < e.nnz) return SDDDST_ERR_CAPACITY;
    cudaMemcpyAsync(host, Lp->d_cval, sizeof(float) * e.nnz, cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("learned export")) return rc;
    if (*Lp->h_err) {
        e.err = "learned preconditioner: a tensor-core product did not complete";
        return SDDDST_ERR_CUDA;
    }
    return 0;
}

void learned_free(Engine &e)
{
    Learned *L = LN(e);
    if (!L) return;
    void *bufs[] = {L->d_w, L->d_nf, L->d_h, L->d_ph, L->d_qh, L->d_agg, L->d_jii, L->d_cval, L->d_crow, L->d_ccnt,
                    L->d_ccol, L->d_cv, L->d_err, L->d_craw, L->d_crawd, L->d_rp0, L->d_col0, L->d_craw0};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (L->h_err) cudaFreeHost(L->h_err);
    learned_train_free(L->train);
    delete L;
    e.learned = nullptr;
}

long learned_weight_count() { return offsets().total; }

} // namespace sd
