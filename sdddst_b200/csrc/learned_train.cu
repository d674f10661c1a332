// Training of the learned preconditioner correction on the device: the
// forward pass of the network (the inference kernels, with every layer's
// node states kept), the loss of sdddst_b200/learned.py (learned_train.py
// trained it in PyTorch before), its gradient by hand-written backward
// kernels, global-norm clipping and Adam on FP32 master weights, and the
// BF16 weights the inference reads refreshed after every step.
//
// Loss for one Jacobian J (at the step size h of a run of the method) with
// its cluster inverse B and k random sign probes Z (n x k):
//   R0 = Z - J B Z,  R = R0 - J C Z,  L = ||R||_F^2 / ||Z||_F^2,
// C the network's correction (C_ij = (c_ij - (1 - s_ij)) A_ij / (J_ii J_jj),
// C_ii = c_ii / J_ii).  Backward:
//   dR = 2 R / (n k),  Gm = -J^T dR,  dC_ij = sum_p Gm_ip Z_jp,
//   dc_ij = dC_ij A_ij / (J_ii J_jj),  dc_ii = dC_ii / J_ii,
// then through the output layer, the three message-passing rounds and the
// input layer.  The per-edge backward runs over the CSR rows twice: once
// in the forward direction (row i collects the gradient of P h_i, and the
// edge weights' gradients), once in the reverse direction (row j collects
// the gradient of Q h_j from the edges (i, j) that gathered it, the edge
// quantities recomputed from row j's own entry of the symmetric pattern), so
// no edge-sized buffer and no atomics are needed.  The node-level products
// are the tensor-core kernels:
//   input gradients  dX[n x NOUT] += dY[n x K] W'   (W' the BF16 weights
//                    transposed into [NOUT][K]; node_gemm_tc's layout),
//   weight gradients dW[128 x N]  = sum_i dY_i (x) X_i over the nodes,
//                    the node dimension as the MMA's K, 128 nodes per step,
//                    per-CTA partials in FP32 reduced in a fixed order,
// both with BF16 operands and FP32 accumulation in tensor memory
// (tcgen05.mma kind::f16, operands staged in shared memory in the no-swizzle
// K-major core-matrix layout, bounded mbarrier waits).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "learned_net.cuh"

namespace sd {

int learned_ensure(Engine &e); // learned.cu

using namespace ln;

namespace {

constexpr int kMaxProbes = 8;
constexpr int kEdgeWarps = 8 * 148 * 4; // fixed grid of the edge backward kernels (per-warp partials)
constexpr int kEdgeCTAs = kEdgeWarps / 8;

__device__ __forceinline__ unsigned hash3(unsigned long long seed, unsigned a, unsigned b)
{
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (a + 1) + 0xBF58476D1CE4E5B9ull * (b + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (unsigned)(z ^ (z >> 31));
}

// Z[p n + i] = +-1
__global__ void probe_kernel(int n, int k, unsigned long long seed, double *__restrict__ Z)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * k) return;
    const int p = (int)(idx / n), i = (int)(idx % n);
    Z[idx] = (hash3(seed, (unsigned)p, (unsigned)i) & 1u) ? 1.0 : -1.0;
}

// Y = J X (trans false) or J^T X (trans true) for k vectors (X[p n + i]),
// J = I + F G with F = diag((1 + d)/2 h), G the CSR (diagonal in slot 0,
// symmetric): J X = X + F (G X), J^T X = X + G (F X).  One warp per row.
template <typename VT>
__global__ void jmul_kernel(int n, int k, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                            const VT *__restrict__ val, const double *__restrict__ dvec, const double *__restrict__ X,
                            double *__restrict__ Y, bool trans, double sign)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    double acc[kMaxProbes];
#pragma unroll
    for (int p = 0; p < kMaxProbes; ++p) acc[p] = 0.0;
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) {
        const int j = col[q];
        double g = (double)val[q];
        if (trans) g *= (1.0 + dvec[j]) * 0.5 * h;
#pragma unroll
        for (int p = 0; p < kMaxProbes; ++p)
            if (p < k) acc[p] += g * X[(long)p * n + j];
    }
    const double fi = trans ? 1.0 : (1.0 + dvec[i]) * 0.5 * h;
#pragma unroll
    for (int p = 0; p < kMaxProbes; ++p) {
        if (p >= k) break;
        const double s = warp_sum(acc[p]);
        if (lane == 0) Y[(long)p * n + i] = sign * (X[(long)p * n + i] + fi * s);
    }
}

// Y = C X for k vectors (C on J's pattern, values cval, diagonal in slot 0)
__global__ void capply_kernel(int n, int k, const int *__restrict__ rowptr, const int *__restrict__ col,
                              const float *__restrict__ cval, const double *__restrict__ X, double *__restrict__ Y)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    double acc[kMaxProbes];
#pragma unroll
    for (int p = 0; p < kMaxProbes; ++p) acc[p] = 0.0;
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) {
        const int j = col[q];
        const double c = (double)cval[q];
#pragma unroll
        for (int p = 0; p < kMaxProbes; ++p)
            if (p < k) acc[p] += c * X[(long)p * n + j];
    }
#pragma unroll
    for (int p = 0; p < kMaxProbes; ++p) {
        if (p >= k) break;
        const double s = warp_sum(acc[p]);
        if (lane == 0) Y[(long)p * n + i] = s;
    }
}

// a = b - c elementwise; partial sums of a^2 per CTA (fixed grid)
__global__ void sub_sq_kernel(long m, const double *__restrict__ b, const double *__restrict__ c,
                              double *__restrict__ a, double *__restrict__ part)
{
    __shared__ double sh[8];
    double s = 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (long)gridDim.x * blockDim.x) {
        const double v = b[t] - c[t];
        a[t] = v;
        s += v * v;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}

// x *= s elementwise
// x *= num / (sum of the np partials in ref): the residual's gradient
// relative to |R0|^2, so every Jacobian's step is scale-free (the loss with B
// alone spans decades over the step sizes a run visits)
__global__ void scale_by_sum_kernel(long m, double num, const double *__restrict__ ref, int np, double *__restrict__ x)
{
    __shared__ double sh[8];
    double r = 0.0;
    for (int b = threadIdx.x; b < np; b += blockDim.x) r += ref[b];
    r = warp_sum(r);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = r;
    __syncthreads();
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
    const double s = tot > 0.0 ? num / tot : 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (long)gridDim.x * blockDim.x) x[t] *= s;
}

// Edge features of the edge (i, j) seen from row i's entry q (the forward
// kernels' definition): e = [t(A_ij), t(A_ji), dx/7c, dy/7c, s_ij], with
// dx = x_j - x_i, dy = y_j - y_i (minimum image); scale = A_ij / (J_ii J_jj).
__device__ __forceinline__ void edge_feat(double g, double di, double dj, double ji, double jj, double xi, double yi,
                                          double xj, double yj, bool same, float inv_pos, float f[kEF], float &sc)
{
    const double aij = di * g, aji = dj * g;
    double dx = xj - xi, dy = yj - yi;
    dx -= rint(dx);
    dy -= rint(dy);
    f[0] = tlogf((float)aij);
    f[1] = tlogf((float)aji);
    f[2] = (float)dx * inv_pos;
    f[3] = (float)dy * inv_pos;
    f[4] = same ? 1.0f : 0.0f;
    sc = (float)(aij / (ji * jj));
}

// dc of every entry: off-diagonal dcraw_q = (sum_p Gm_ip Z_jp) A_ij / (J_ii J_jj),
// diagonal dcrawd_i = (sum_p Gm_ip Z_ip) / J_ii.  One warp per row.
template <typename VT>
__global__ void dc_kernel(int n, int k, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                          const VT *__restrict__ val, const double *__restrict__ dvec,
                          const double *__restrict__ jii, const double *__restrict__ Gm,
                          const double *__restrict__ Z, float *__restrict__ dcraw, float *__restrict__ dcrawd)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    double gi[kMaxProbes];
#pragma unroll
    for (int p = 0; p < kMaxProbes; ++p) gi[p] = p < k ? Gm[(long)p * n + i] : 0.0;
    const double di = (1.0 + dvec[i]) * 0.5 * h, ji = jii[i];
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) {
        const int j = col[q];
        double s = 0.0;
#pragma unroll
        for (int p = 0; p < kMaxProbes; ++p)
            if (p < k) s += gi[p] * Z[(long)p * n + j];
        if (j == i) dcrawd[i] = (float)(s / ji);
        else dcraw[q] = (float)(s * (di * (double)val[q]) / (ji * jii[j]));
    }
}

// ---- per-edge backward.  A fixed grid of kEdgeWarps warps walks the rows
// (warp w takes rows w, w + kEdgeWarps, ...); lane l holds channels l and
// l + 32; the edges of a row are taken 32 at a time, lane t computing edge
// t's features and scalars, then all lanes walking the 32 edges (shuffles).
// Per-warp partial weight gradients go to part[warp][...], summed later in a
// fixed order.

// Output layer, forward direction: row i collects dpo_i; partials of dRo
// (64 x 5), dwo (64) and dbo.
template <typename VT>
__global__ void __launch_bounds__(256) oedge_fwd_kernel(
    int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col, const VT *__restrict__ val,
    const double *__restrict__ dvec, const double *__restrict__ jii, const double *__restrict__ x,
    const double *__restrict__ y, const int *__restrict__ blk, double cutoff, const float *__restrict__ po,
    const __nv_bfloat16 *__restrict__ qo, const __nv_bfloat16 *__restrict__ w, long oRo, long owo,
    const float *__restrict__ dcraw, float *__restrict__ dpo, float *__restrict__ part)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int c0 = lane, c1 = lane + 32;
    float r0[kEF], r1[kEF];
#pragma unroll
    for (int f = 0; f < kEF; ++f) {
        r0[f] = bf(w, oRo + c0 * kEF + f);
        r1[f] = bf(w, oRo + c1 * kEF + f);
    }
    const float wo0 = bf(w, owo + c0), wo1 = bf(w, owo + c1);
    const float inv_pos = (float)(1.0 / (kPosScale * cutoff));
    float dR0[kEF] = {0, 0, 0, 0, 0}, dR1[kEF] = {0, 0, 0, 0, 0};
    float dwo0 = 0.0f, dwo1 = 0.0f, dbo = 0.0f;
    for (int i = gw; i < n; i += kEdgeWarps) {
        const float p0 = po[(long)i * kH + c0], p1 = po[(long)i * kH + c1];
        const double di = (1.0 + dvec[i]) * 0.5 * h, ji = jii[i], xi = x[i], yi = y[i];
        const int bi = blk[i];
        float g0 = 0.0f, g1 = 0.0f;
        const int qs = rowptr[i], qe = rowptr[i + 1];
        for (int q0 = qs; q0 < qe; q0 += 32) {
            const int q = q0 + lane;
            int j = -1;
            float fe[kEF] = {0, 0, 0, 0, 0}, sc = 0.0f, dcr = 0.0f;
            if (q < qe) {
                j = col[q];
                if (j != i) {
                    edge_feat((double)val[q], di, (1.0 + dvec[j]) * 0.5 * h, ji, jii[j], xi, yi, x[j], y[j],
                              blk[j] == bi, inv_pos, fe, sc);
                    dcr = dcraw[q];
                } else {
                    j = -1;
                }
            }
#pragma unroll 4
            for (int t = 0; t < 32; ++t) {
                const int jt = __shfl_sync(0xffffffffu, j, t);
                float f[kEF];
#pragma unroll
                for (int u = 0; u < kEF; ++u) f[u] = __shfl_sync(0xffffffffu, fe[u], t);
                const float d = __shfl_sync(0xffffffffu, dcr, t);
                if (jt < 0) continue;
                float a = p0 + __bfloat162float(qo[(long)jt * kH + c0]);
                float b = p1 + __bfloat162float(qo[(long)jt * kH + c1]);
#pragma unroll
                for (int u = 0; u < kEF; ++u) {
                    a = fmaf(r0[u], f[u], a);
                    b = fmaf(r1[u], f[u], b);
                }
                const float ga = a > 0.0f ? d * wo0 : 0.0f, gb = b > 0.0f ? d * wo1 : 0.0f;
                g0 += ga;
                g1 += gb;
#pragma unroll
                for (int u = 0; u < kEF; ++u) {
                    dR0[u] = fmaf(ga, f[u], dR0[u]);
                    dR1[u] = fmaf(gb, f[u], dR1[u]);
                }
                dwo0 = fmaf(d, fmaxf(a, 0.0f), dwo0);
                dwo1 = fmaf(d, fmaxf(b, 0.0f), dwo1);
                if (lane == 0) dbo += d;
            }
        }
        dpo[(long)i * kH + c0] = g0;
        dpo[(long)i * kH + c1] = g1;
    }
    float *pp = part + (long)gw * (kH * kEF + kH + 1);
#pragma unroll
    for (int u = 0; u < kEF; ++u) {
        pp[c0 * kEF + u] = dR0[u];
        pp[c1 * kEF + u] = dR1[u];
    }
    pp[kH * kEF + c0] = dwo0;
    pp[kH * kEF + c1] = dwo1;
    if (lane == 0) pp[kH * kEF + kH] = dbo;
}

// Output layer, reverse direction: row j collects dqo_j = sum over the
// edges (i, j) of dc_ij w_o [relu'] with dc_ij = (sum_p Gm_ip Z_jp) A_ij / (J_ii J_jj)
// recomputed here.
template <typename VT>
__global__ void __launch_bounds__(256) oedge_rev_kernel(
    int n, int k, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
    const VT *__restrict__ val, const double *__restrict__ dvec, const double *__restrict__ jii,
    const double *__restrict__ x, const double *__restrict__ y, const int *__restrict__ blk, double cutoff,
    const float *__restrict__ po, const __nv_bfloat16 *__restrict__ qo, const __nv_bfloat16 *__restrict__ w,
    long oRo, long owo, const double *__restrict__ Gm, const double *__restrict__ Z, float *__restrict__ dqo)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int c0 = lane, c1 = lane + 32;
    float r0[kEF], r1[kEF];
#pragma unroll
    for (int f = 0; f < kEF; ++f) {
        r0[f] = bf(w, oRo + c0 * kEF + f);
        r1[f] = bf(w, oRo + c1 * kEF + f);
    }
    const float wo0 = bf(w, owo + c0), wo1 = bf(w, owo + c1);
    const float inv_pos = (float)(1.0 / (kPosScale * cutoff));
    for (int j = gw; j < n; j += kEdgeWarps) {
        const float q0v = __bfloat162float(qo[(long)j * kH + c0]), q1v = __bfloat162float(qo[(long)j * kH + c1]);
        const double dj = (1.0 + dvec[j]) * 0.5 * h, jj = jii[j], xj = x[j], yj = y[j];
        const int bj = blk[j];
        double zj[kMaxProbes];
#pragma unroll
        for (int p = 0; p < kMaxProbes; ++p) zj[p] = p < k ? Z[(long)p * n + j] : 0.0;
        float g0 = 0.0f, g1 = 0.0f;
        const int qs = rowptr[j], qe = rowptr[j + 1];
        for (int qb = qs; qb < qe; qb += 32) {
            const int q = qb + lane;
            int i = -1;
            float fe[kEF] = {0, 0, 0, 0, 0}, dcr = 0.0f;
            if (q < qe) {
                i = col[q];
                if (i != j) {
                    float sc;
                    const double di = (1.0 + dvec[i]) * 0.5 * h;
                    edge_feat((double)val[q], di, dj, jii[i], jj, x[i], y[i], xj, yj, blk[i] == bj, inv_pos, fe, sc);
                    double s = 0.0;
#pragma unroll
                    for (int p = 0; p < kMaxProbes; ++p)
                        if (p < k) s += Gm[(long)p * n + i] * zj[p];
                    dcr = (float)s * sc;
                } else {
                    i = -1;
                }
            }
#pragma unroll 4
            for (int t = 0; t < 32; ++t) {
                const int it = __shfl_sync(0xffffffffu, i, t);
                float f[kEF];
#pragma unroll
                for (int u = 0; u < kEF; ++u) f[u] = __shfl_sync(0xffffffffu, fe[u], t);
                const float d = __shfl_sync(0xffffffffu, dcr, t);
                if (it < 0) continue;
                float a = po[(long)it * kH + c0] + q0v, b = po[(long)it * kH + c1] + q1v;
#pragma unroll
                for (int u = 0; u < kEF; ++u) {
                    a = fmaf(r0[u], f[u], a);
                    b = fmaf(r1[u], f[u], b);
                }
                if (a > 0.0f) g0 = fmaf(d, wo0, g0);
                if (b > 0.0f) g1 = fmaf(d, wo1, g1);
            }
        }
        dqo[(long)j * kH + c0] = g0;
        dqo[(long)j * kH + c1] = g1;
    }
}

// Message layer, forward direction: with g_i = da_i / deg_i, row i collects
// dph_i,c = g_i,c #{edges with pre_c > 0}; partials of dR (64 x 5).
template <typename VT>
__global__ void __launch_bounds__(256) ledge_fwd_kernel(
    int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col, const VT *__restrict__ val,
    const double *__restrict__ dvec, const double *__restrict__ jii, const double *__restrict__ x,
    const double *__restrict__ y, const int *__restrict__ blk, double cutoff, const float *__restrict__ ph,
    const __nv_bfloat16 *__restrict__ qh, const __nv_bfloat16 *__restrict__ w, long oR,
    const float *__restrict__ da, float *__restrict__ dph, float *__restrict__ part)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int c0 = lane, c1 = lane + 32;
    float r0[kEF], r1[kEF];
#pragma unroll
    for (int f = 0; f < kEF; ++f) {
        r0[f] = bf(w, oR + c0 * kEF + f);
        r1[f] = bf(w, oR + c1 * kEF + f);
    }
    const float inv_pos = (float)(1.0 / (kPosScale * cutoff));
    float dR0[kEF] = {0, 0, 0, 0, 0}, dR1[kEF] = {0, 0, 0, 0, 0};
    for (int i = gw; i < n; i += kEdgeWarps) {
        const int qs = rowptr[i], qe = rowptr[i + 1];
        const float inv_deg = 1.0f / (float)max(qe - qs - 1, 1);
        const float ga = da[(long)i * kH + c0] * inv_deg, gb = da[(long)i * kH + c1] * inv_deg;
        const float p0 = ph[(long)i * kH + c0], p1 = ph[(long)i * kH + c1];
        const double di = (1.0 + dvec[i]) * 0.5 * h, ji = jii[i], xi = x[i], yi = y[i];
        const int bi = blk[i];
        float n0 = 0.0f, n1 = 0.0f, fs0[kEF] = {0, 0, 0, 0, 0}, fs1[kEF] = {0, 0, 0, 0, 0};
        for (int qb = qs; qb < qe; qb += 32) {
            const int q = qb + lane;
            int j = -1;
            float fe[kEF] = {0, 0, 0, 0, 0}, sc;
            if (q < qe) {
                j = col[q];
                if (j != i)
                    edge_feat((double)val[q], di, (1.0 + dvec[j]) * 0.5 * h, ji, jii[j], xi, yi, x[j], y[j],
                              blk[j] == bi, inv_pos, fe, sc);
                else
                    j = -1;
            }
#pragma unroll 4
            for (int t = 0; t < 32; ++t) {
                const int jt = __shfl_sync(0xffffffffu, j, t);
                float f[kEF];
#pragma unroll
                for (int u = 0; u < kEF; ++u) f[u] = __shfl_sync(0xffffffffu, fe[u], t);
                if (jt < 0) continue;
                float a = p0 + __bfloat162float(qh[(long)jt * kH + c0]);
                float b = p1 + __bfloat162float(qh[(long)jt * kH + c1]);
#pragma unroll
                for (int u = 0; u < kEF; ++u) {
                    a = fmaf(r0[u], f[u], a);
                    b = fmaf(r1[u], f[u], b);
                }
                if (a > 0.0f) {
                    n0 += 1.0f;
#pragma unroll
                    for (int u = 0; u < kEF; ++u) fs0[u] += f[u];
                }
                if (b > 0.0f) {
                    n1 += 1.0f;
#pragma unroll
                    for (int u = 0; u < kEF; ++u) fs1[u] += f[u];
                }
            }
        }
        dph[(long)i * kH + c0] = ga * n0;
        dph[(long)i * kH + c1] = gb * n1;
#pragma unroll
        for (int u = 0; u < kEF; ++u) {
            dR0[u] = fmaf(ga, fs0[u], dR0[u]);
            dR1[u] = fmaf(gb, fs1[u], dR1[u]);
        }
    }
    float *pp = part + (long)gw * (kH * kEF);
#pragma unroll
    for (int u = 0; u < kEF; ++u) {
        pp[c0 * kEF + u] = dR0[u];
        pp[c1 * kEF + u] = dR1[u];
    }
}

// Message layer, reverse direction: row j collects dqh_j,c = sum over the
// edges (i, j) of g_i,c [ph_i,c + qh_j,c + R_c e_ij > 0].
template <typename VT>
__global__ void __launch_bounds__(256) ledge_rev_kernel(
    int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col, const VT *__restrict__ val,
    const double *__restrict__ dvec, const double *__restrict__ jii, const double *__restrict__ x,
    const double *__restrict__ y, const int *__restrict__ blk, double cutoff, const float *__restrict__ ph,
    const __nv_bfloat16 *__restrict__ qh, const __nv_bfloat16 *__restrict__ w, long oR,
    const float *__restrict__ da, float *__restrict__ dqh)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int c0 = lane, c1 = lane + 32;
    float r0[kEF], r1[kEF];
#pragma unroll
    for (int f = 0; f < kEF; ++f) {
        r0[f] = bf(w, oR + c0 * kEF + f);
        r1[f] = bf(w, oR + c1 * kEF + f);
    }
    const float inv_pos = (float)(1.0 / (kPosScale * cutoff));
    for (int j = gw; j < n; j += kEdgeWarps) {
        const float q0v = __bfloat162float(qh[(long)j * kH + c0]), q1v = __bfloat162float(qh[(long)j * kH + c1]);
        const double dj = (1.0 + dvec[j]) * 0.5 * h, jj = jii[j], xj = x[j], yj = y[j];
        const int bj = blk[j];
        float g0 = 0.0f, g1 = 0.0f;
        const int qs = rowptr[j], qe = rowptr[j + 1];
        for (int qb = qs; qb < qe; qb += 32) {
            const int q = qb + lane;
            int i = -1;
            float fe[kEF] = {0, 0, 0, 0, 0}, inv_deg = 0.0f;
            if (q < qe) {
                i = col[q];
                if (i != j) {
                    float sc;
                    edge_feat((double)val[q], (1.0 + dvec[i]) * 0.5 * h, dj, jii[i], jj, x[i], y[i], xj, yj,
                              blk[i] == bj, inv_pos, fe, sc);
                    inv_deg = 1.0f / (float)max(rowptr[i + 1] - rowptr[i] - 1, 1);
                } else {
                    i = -1;
                }
            }
#pragma unroll 4
            for (int t = 0; t < 32; ++t) {
                const int it = __shfl_sync(0xffffffffu, i, t);
                float f[kEF];
#pragma unroll
                for (int u = 0; u < kEF; ++u) f[u] = __shfl_sync(0xffffffffu, fe[u], t);
                const float idg = __shfl_sync(0xffffffffu, inv_deg, t);
                if (it < 0) continue;
                float a = ph[(long)it * kH + c0] + q0v, b = ph[(long)it * kH + c1] + q1v;
#pragma unroll
                for (int u = 0; u < kEF; ++u) {
                    a = fmaf(r0[u], f[u], a);
                    b = fmaf(r1[u], f[u], b);
                }
                if (a > 0.0f) g0 = fmaf(da[(long)it * kH + c0], idg, g0);
                if (b > 0.0f) g1 = fmaf(da[(long)it * kH + c1], idg, g1);
            }
        }
        dqh[(long)j * kH + c0] = g0;
        dqh[(long)j * kH + c1] = g1;
    }
}

// sum over the kEdgeWarps partial rows of width m into g[off + c] (fixed order)
__global__ void part_reduce_kernel(int rows, int m, const float *__restrict__ part, float *__restrict__ g, long off)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += part[(long)r * m + c];
    g[off + c] += s;
}

// column sums of X (n x 64) into g[off + c] (one CTA per column, fixed order)
__global__ void colsum_kernel(int n, const float *__restrict__ X, float *__restrict__ g, long off)
{
    __shared__ float sh[8];
    const int c = blockIdx.x;
    float s = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += X[(long)i * kH + c];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        g[off + c] += t;
    }
}

// diagonal output: dwd_c = sum_i dcrawd_i h_ic, dbd = sum_i dcrawd_i (one CTA
// per channel, c = 64: the bias), and dh_i += dcrawd_i w_d (separate kernel)
__global__ void dout_w_kernel(int n, const float *__restrict__ dcrawd, const float *__restrict__ hin,
                              float *__restrict__ g, long owd, long owdb)
{
    __shared__ float sh[8];
    const int c = blockIdx.x;
    float s = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += dcrawd[i] * (c < kH ? hin[(long)i * kH + c] : 1.0f);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        g[c < kH ? owd + c : owdb] += t;
    }
}

__global__ void dout_h_kernel(int n, const float *__restrict__ dcrawd, const __nv_bfloat16 *__restrict__ w, long owd,
                              float *__restrict__ dh)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * kH) return;
    dh[idx] += dcrawd[idx >> 6] * bf(w, owd + (idx & 63));
}

// du = dh [h_next > h_prev] (the update's ReLU is active where it added)
__global__ void relu_mask_kernel(long m, const float *__restrict__ dh, const float *__restrict__ hn,
                                 const float *__restrict__ hp, float *__restrict__ du)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) du[t] = hn[t] > hp[t] ? dh[t] : 0.0f;
}

// input layer: d = dh0 [h0 > 0]; dW_in[c][f] = sum_i d_ic nf_if, db_in = sum_i d_ic
// (one CTA per output channel)
__global__ void din_kernel(int n, const float *__restrict__ dh0, const float *__restrict__ h0,
                           const float *__restrict__ nf, float *__restrict__ g, long oin_w, long oin_b)
{
    __shared__ float sh[5][8];
    const int c = blockIdx.x;
    float s[5] = {0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const long idx = (long)i * kH + c;
        const float d = h0[idx] > 0.0f ? dh0[idx] : 0.0f;
#pragma unroll
        for (int f = 0; f < kNF; ++f) s[f] = fmaf(d, nf[4 * i + f], s[f]);
        s[4] += d;
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        const float v = warp_sum(s[f]);
        if ((threadIdx.x & 31) == 0) sh[f][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[threadIdx.x][w];
        if (threadIdx.x < kNF) g[oin_w + c * kNF + threadIdx.x] += t;
        else g[oin_b + c] += t;
    }
}

// Adam on the FP32 master weights after global-norm clipping; the BF16
// weights of the inference refreshed (round to nearest even).  One CTA
// computes the norm first (norm_kernel), then every thread one weight.
__global__ void norm_kernel(long m, const float *__restrict__ g, float *__restrict__ out)
{
    __shared__ double sh[32];
    double s = 0.0;
    for (long t = threadIdx.x; t < m; t += blockDim.x) s += (double)g[t] * g[t];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        out[0] = (float)sqrt(t);
    }
}

__global__ void adam_kernel(long m, float *__restrict__ W, float *__restrict__ M, float *__restrict__ V,
                            const float *__restrict__ g, const float *__restrict__ gnorm, float clip, float lr,
                            float b1, float b2, float eps, float c1, float c2, __nv_bfloat16 *__restrict__ wbf)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const float nrm = gnorm[0];
    const float s = nrm > clip ? clip / (nrm + 1e-6f) : 1.0f;
    const float gt = g[t] * s;
    const float mt = b1 * M[t] + (1.0f - b1) * gt, vt = b2 * V[t] + (1.0f - b2) * gt * gt;
    M[t] = mt;
    V[t] = vt;
    const float wt = W[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    W[t] = wt;
    wbf[t] = __float2bfloat16_rn(wt);
}

// ---- tensor-core products of the backward pass (tcgen05.mma kind::f16:
// BF16 operands staged in shared memory, FP32 accumulation in tensor memory)

// byte offset of element (r, k) of an R x K BF16 tile in the no-swizzle
// K-major core-matrix layout (8 rows x 16 bytes per core matrix, K-adjacent
// core matrices 128 bytes apart, 8-row groups K/8 x 128 bytes apart)
__device__ __forceinline__ unsigned tile_off(int r, int k, int K)
{
    return (unsigned)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ unsigned long long mma_desc(unsigned addr, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)(128u >> 4) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ unsigned s32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// bounded wait on an mbarrier phase; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned mb, unsigned parity)
{
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(mb), "r"(parity)
                     : "memory");
        if (!done && it > 32) __nanosleep(64);
    }
    return done != 0;
}

__device__ __forceinline__ void issue_mmas(unsigned tmem, unsigned a0, unsigned b0, int ksteps, unsigned sbo,
                                           unsigned idesc, bool first)
{
    for (int t = 0; t < ksteps; ++t) {
        const unsigned long long ad = mma_desc(a0 + 256u * t, sbo), bd = mma_desc(b0 + 256u * t, sbo);
        const unsigned acc = (first && t == 0) ? 0u : 1u;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                     "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    }
}

// out[n x NOUT] (+)= X[n x K] Wt^T over 128-node tiles; X = [X0 | X1] (n x 64
// each, X1 when K = 128), out = [out0 | out1] (out1 when NOUT = 128), Wt the
// BF16 [NOUT][K] matrix.  acc0 / acc1: add to out0 / out1 (else overwrite).
template <int K, int NOUT>
__global__ void __launch_bounds__(128) tc_dx_kernel(int n, const float *__restrict__ X0, const float *__restrict__ X1,
                                                    const __nv_bfloat16 *__restrict__ Wt, float *__restrict__ out0,
                                                    float *__restrict__ out1, bool acc0, bool acc1,
                                                    int *__restrict__ err)
{
    constexpr unsigned kSBO = (K / 8) * 128;
    constexpr unsigned kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(NOUT >> 3) << 17) | ((128u >> 4) << 24);
    extern __shared__ __align__(1024) unsigned char smem_dx[];
    unsigned char *As = smem_dx, *Bs = smem_dx + 128 * K * 2;
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, i0 = blockIdx.x * 128;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s32(&tslot)),
                     "r"((unsigned)NOUT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s32(&mbar)), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    {
        const int i = i0 + tid;
        for (int k = 0; k < K; k += 2) {
            float a = 0.0f, b = 0.0f;
            if (i < n) {
                const float *src = k < 64 ? X0 : X1;
                a = src[(long)i * 64 + (k & 63)];
                b = src[(long)i * 64 + ((k + 1) & 63)];
            }
            const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
            *reinterpret_cast<__nv_bfloat162 *>(As + tile_off(tid, k, K)) = v;
        }
        for (int idx = tid; idx < NOUT * K; idx += 128) {
            const int c = idx / K, k = idx % K;
            *reinterpret_cast<__nv_bfloat16 *>(Bs + tile_off(c, k, K)) = Wt[idx];
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tslot, mb = s32(&mbar);
    if (tid == 0) {
        issue_mmas(tmem, s32(As), s32(Bs), K / 16, kSBO, kIdesc, true);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb) : "memory");
    }
    const bool done = mbar_wait(mb, 0u);
    if (!done && lane == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__all_sync(0xffffffffu, done)) {
        const int i = i0 + warp * 32 + lane;
        const unsigned base = (unsigned)(warp * 32) << 16;
#pragma unroll
        for (int c0 = 0; c0 < NOUT; c0 += 16) {
            unsigned v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + base + (unsigned)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (i < n) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int c = c0 + q;
                    const float d = __uint_as_float(v[q]);
                    float *o = c < 64 ? out0 : out1;
                    const bool ac = c < 64 ? acc0 : acc1;
                    const long at = (long)i * 64 + (c & 63);
                    o[at] = ac ? o[at] + d : d;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)NOUT));
}

// Weight gradient D[128 x N] = sum over the nodes of A_i (x) B_i, with
// A_i = [A0_i; A1_i] (64 + 64 channels; zeros for a missing A1) and
// B_i = [B0_i; B1_i] (N = 64: B0 only) rounded to BF16; the node dimension is
// the MMA's K, 128 nodes per chunk (8 MMAs of K = 16).  CTA b takes chunks
// b, b + grid, ... and writes its FP32 partial to part[b][128][N].
template <int N>
__global__ void __launch_bounds__(128) tc_wgrad_kernel(int n, const float *__restrict__ A0,
                                                       const float *__restrict__ A1, const float *__restrict__ B0,
                                                       const float *__restrict__ B1, float *__restrict__ part,
                                                       int *__restrict__ err)
{
    constexpr unsigned kSBO = (128 / 8) * 128;
    constexpr unsigned kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((128u >> 4) << 24);
    extern __shared__ __align__(1024) unsigned char smem_wg[];
    unsigned char *As = smem_wg, *Bs = smem_wg + 128 * 128 * 2;
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s32(&tslot)),
                     "r"((unsigned)N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s32(&mbar)), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tslot, mb = s32(&mbar);
    const int chunks = (n + 127) / 128;
    bool ok = true, first = true;
    unsigned phase = 0;
    for (int c = blockIdx.x; c < chunks && ok; c += gridDim.x) {
        // thread t stages node c*128 + t: column t of A (128 channels) and of B
        const int i = c * 128 + tid;
        for (int r = 0; r < 128; ++r) {
            float a = 0.0f;
            if (i < n) a = r < 64 ? A0[(long)i * 64 + r] : (A1 ? A1[(long)i * 64 + r - 64] : 0.0f);
            *reinterpret_cast<__nv_bfloat16 *>(As + tile_off(r, tid, 128)) = __float2bfloat16_rn(a);
        }
        for (int r = 0; r < N; ++r) {
            float b = 0.0f;
            if (i < n) b = r < 64 ? B0[(long)i * 64 + r] : B1[(long)i * 64 + r - 64];
            *reinterpret_cast<__nv_bfloat16 *>(Bs + tile_off(r, tid, 128)) = __float2bfloat16_rn(b);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            issue_mmas(tmem, s32(As), s32(Bs), 8, kSBO, kIdesc, first);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        first = false;
        const bool done = mbar_wait(mb, phase);
        phase ^= 1u;
        ok = __syncthreads_and(done) != 0; // the tiles are overwritten only after the MMAs read them
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        const int r = warp * 32 + lane;
        const unsigned base = (unsigned)(warp * 32) << 16;
        float *pp = part + ((long)blockIdx.x * 128 + r) * N;
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            unsigned v[16];
            if (first) { // no chunk for this CTA: a zero partial
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] = 0u;
            } else {
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
                             "%11, %12, %13, %14, %15}, [%16];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                               "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                             : "r"(tmem + base + (unsigned)c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) pp[c0 + q] = __uint_as_float(v[q]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)N));
}

// g[oA0 + r N + c] += sum_b part[b][r][c] (r < 64), g[oA1 + (r - 64) N + c] (r >= 64, when oA1 >= 0)
__global__ void wgrad_reduce_kernel(int blocks, int N, const float *__restrict__ part, float *__restrict__ g, long oA0,
                                    long oA1)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 128 * N) return;
    const int r = t / N, c = t % N;
    if (r >= 64 && oA1 < 0) return;
    float s = 0.0f;
    for (int b = 0; b < blocks; ++b) s += part[((long)b * 128 + r) * N + c];
    g[(r < 64 ? oA0 + (long)r * N : oA1 + (long)(r - 64) * N) + c] += s;
}

// Wt for the input gradients from the BF16 weights:
//   PQ (NOUT 64, K 128): Wt[k][o] = o < 64 ? P[o][k] : Q[o - 64][k]
//   U  (NOUT 128, K 64): Wt[k][o] = U[o][k] (U is [64][128])
__global__ void transpose_pq_kernel(const __nv_bfloat16 *__restrict__ w, long oP, long oQ,
                                    __nv_bfloat16 *__restrict__ wt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 64 * 128) return;
    const int k = t / 128, o = t % 128;
    wt[t] = o < 64 ? w[oP + (long)o * 64 + k] : w[oQ + (long)(o - 64) * 64 + k];
}

__global__ void transpose_u_kernel(const __nv_bfloat16 *__restrict__ w, long oU, __nv_bfloat16 *__restrict__ wt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 128 * 64) return;
    const int k = t / 64, o = t % 64;
    wt[t] = w[oU + (long)o * 128 + k];
}

struct Train {
    int n = 0;
    long nw = 0;          // weights
    float *W = nullptr, *M = nullptr, *V = nullptr, *g = nullptr, *gnorm = nullptr;
    long steps = 0;
    double *dvec = nullptr, *Z = nullptr, *BZ = nullptr, *R0 = nullptr, *T1 = nullptr, *T2 = nullptr,
           *dpart = nullptr, *h_loss = nullptr;
    float *h[kLayers + 1] = {}, *ph[kLayers] = {}, *a[kLayers] = {};
    __nv_bfloat16 *qh[kLayers] = {};
    float *po = nullptr, *dh = nullptr, *dY0 = nullptr, *dY1 = nullptr, *da = nullptr, *du = nullptr,
          *dcraw = nullptr, *dcrawd = nullptr, *epart = nullptr, *wpart = nullptr;
    __nv_bfloat16 *qo = nullptr, *wt_pq = nullptr, *wt_u = nullptr;
    long dcraw_cap = 0;
};

constexpr int kWgradCTAs = 148;
constexpr int kSubCTAs = 256;

Train *TR(Engine &e) { return e.learned ? static_cast<Train *>(LN(e)->train) : nullptr; }

template <typename T> bool dmalloc(T **p, size_t count)
{
    return cudaMalloc(p, sizeof(T) * (count ? count : 1)) == cudaSuccess;
}

int train_alloc(Engine &e, Train &T)
{
    const size_t n = (size_t)e.n, nh = n * kH;
    T.n = e.n;
    T.nw = offsets().total;
    bool ok = dmalloc(&T.W, T.nw) && dmalloc(&T.M, T.nw) && dmalloc(&T.V, T.nw) && dmalloc(&T.g, T.nw) &&
              dmalloc(&T.gnorm, 1) && dmalloc(&T.dvec, n) && dmalloc(&T.Z, n * kMaxProbes) &&
              dmalloc(&T.BZ, n * kMaxProbes) && dmalloc(&T.R0, n * kMaxProbes) && dmalloc(&T.T1, n * kMaxProbes) &&
              dmalloc(&T.T2, n * kMaxProbes) && dmalloc(&T.dpart, 2 * kSubCTAs) &&
              cudaMallocHost(&T.h_loss, sizeof(double) * 2) == cudaSuccess;
    for (int l = 0; l <= kLayers && ok; ++l) ok = dmalloc(&T.h[l], nh);
    for (int l = 0; l < kLayers && ok; ++l) ok = dmalloc(&T.ph[l], nh) && dmalloc(&T.a[l], nh) && dmalloc(&T.qh[l], nh);
    ok = ok && dmalloc(&T.po, nh) && dmalloc(&T.qo, nh) && dmalloc(&T.dh, nh) && dmalloc(&T.dY0, nh) &&
         dmalloc(&T.dY1, nh) && dmalloc(&T.da, nh) && dmalloc(&T.du, nh) && dmalloc(&T.dcrawd, n) &&
         dmalloc(&T.epart, (size_t)kEdgeWarps * (kH * kEF + kH + 1)) &&
         dmalloc(&T.wpart, (size_t)kWgradCTAs * 128 * 128) && dmalloc(&T.wt_pq, 64 * 128) && dmalloc(&T.wt_u, 128 * 64);
    if (!ok) {
        e.err = "learned training: out of device memory";
        return SDDDST_ERR_NOMEM;
    }
    cudaMemsetAsync(T.M, 0, sizeof(float) * T.nw, e.st);
    cudaMemsetAsync(T.V, 0, sizeof(float) * T.nw, e.st);
    return 0;
}

void set_attrs()
{
    static bool done[256] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev > 255 || done[dev]) return;
    cudaFuncSetAttribute(tc_dx_kernel<128, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(tc_dx_kernel<64, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(tc_wgrad_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(tc_wgrad_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
    done[dev] = true;
}

} // namespace

void learned_train_free(void *p)
{
    Train *T = static_cast<Train *>(p);
    if (!T) return;
    void *bufs[] = {T->W, T->M, T->V, T->g, T->gnorm, T->dvec, T->Z, T->BZ, T->R0, T->T1, T->T2, T->dpart, T->po,
                    T->qo, T->dh, T->dY0, T->dY1, T->da, T->du, T->dcraw, T->dcrawd, T->epart, T->wpart, T->wt_pq,
                    T->wt_u};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (int l = 0; l <= kLayers; ++l)
        if (T->h[l]) cudaFree(T->h[l]);
    for (int l = 0; l < kLayers; ++l) {
        if (T->ph[l]) cudaFree(T->ph[l]);
        if (T->a[l]) cudaFree(T->a[l]);
        if (T->qh[l]) cudaFree(T->qh[l]);
    }
    if (T->h_loss) cudaFreeHost(T->h_loss);
    delete T;
}

// Starts training from the FP32 weights W0 (count = the flat weight count);
// the BF16 weights of the inference are set to their rounding.
int learned_train_init(Engine &e, const float *W0, long count)
{
    if (count != offsets().total) {
        e.err = "learned training: expected " + std::to_string(offsets().total) + " weights";
        return SDDDST_ERR_INVALID;
    }
    if (int rc = learned_ensure(e)) return rc;
    Learned &L = *LN(e);
    if (L.train) {
        learned_train_free(L.train);
        L.train = nullptr;
    }
    Train *T = new Train();
    L.train = T;
    if (int rc = train_alloc(e, *T)) return rc;
    cudaMemcpyAsync(T->W, W0, sizeof(float) * count, cudaMemcpyHostToDevice, e.st);
    std::vector<unsigned short> bf(count);
    for (long t = 0; t < count; ++t) {
        unsigned u;
        std::memcpy(&u, &W0[t], 4);
        bf[t] = (unsigned short)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
    }
    return learned_set_weights(e, bf.data(), count);
}

// One training step on J(h) at the accepted configuration: k probes from
// `seed`, loss and gradient, then (apply) clipping and an Adam step with
// learning rate lr.  loss (optional, 2 doubles) receives ||R0||^2 / ||Z||^2
// (B alone) and ||R||^2 / ||Z||^2 (B + C) before the update; grad (optional,
// host, count floats) the unclipped gradient.
template <typename VT>
int train_step_impl(Engine &e, const VT *val, double h, int k, double lr, unsigned long long seed, bool apply,
                    double *loss, float *grad)
{
    Learned &L = *LN(e);
    Train &T = *TR(e);
    const WeightOffsets &o = L.off;
    const int n = e.n;
    cudaStream_t st = e.st;
    set_attrs();
    const unsigned wrows = (unsigned)((n + 7) / 8);
    const unsigned nt = (unsigned)(((long)n * kH + 255) / 256);
    const long nk = (long)n * k;
    const double *x = e.d_x0;
    // J(h), d, the cluster inverse B, features
    if (int rc = e.assemble(x)) return rc;
    launch_make_dvec(e, h, T.dvec, st);
    if (int rc = precond_build(e, e.pc, h, T.dvec, true)) return rc;
    if (e.nnz > T.dcraw_cap) {
        if (T.dcraw) cudaFree(T.dcraw);
        T.dcraw = nullptr;
        T.dcraw_cap = 0;
        if (!dmalloc(&T.dcraw, (size_t)e.nnz + e.nnz / 8)) {
            e.err = "learned training: out of device memory";
            return SDDDST_ERR_NOMEM;
        }
        T.dcraw_cap = e.nnz + e.nnz / 8;
    }
    if (e.nnz > L.cval_cap) {
        if (L.d_cval) cudaFree(L.d_cval);
        if (L.d_craw) cudaFree(L.d_craw);
        L.d_cval = L.d_craw = nullptr;
        L.cval_cap = 0;
        const long cap = e.nnz + e.nnz / 8;
        if (!dmalloc(&L.d_cval, cap) || !dmalloc(&L.d_craw, cap)) {
            e.err = "learned training: out of device memory";
            return SDDDST_ERR_NOMEM;
        }
        L.cval_cap = cap;
    }
    L.prev_valid = false; // d_craw now receives this step's forward: nothing to remap from
    feat_kernel<VT><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, e.d_gdiag, T.dvec, L.d_nf, L.d_jii);
    // probes, R0 = Z - J B Z
    probe_kernel<<<(unsigned)((nk + 255) / 256), 256, 0, st>>>(n, k, seed, T.Z);
    for (int p = 0; p < k; ++p) precond_apply(e, e.pc, T.Z + (long)p * n, T.BZ + (long)p * n);
    jmul_kernel<VT><<<wrows, 256, 0, st>>>(n, k, h, e.d_rowptr, e.d_col, val, T.dvec, T.BZ, T.T1, false, 1.0);
    sub_sq_kernel<<<kSubCTAs, 256, 0, st>>>(nk, T.Z, T.T1, T.R0, T.dpart);
    // forward, every layer's node states kept
    const int *blk = e.pc.blk_of;
    node_in_kernel<<<nt, 256, 0, st>>>(n, L.d_nf, L.d_w, o.in_w, o.in_b, T.h[0]);
    for (int l = 0; l < kLayers; ++l) {
        launch_node_proj_tc(n, T.h[l], L.d_w, o.P[l], o.Pb[l], o.Q[l], T.ph[l], T.qh[l], L.d_err, st);
        edge_kernel<VT, false><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y, blk,
                                                      e.cutoff, T.ph[l], T.qh[l], L.d_w, o.R[l], 0, 0, T.a[l],
                                                      nullptr, nullptr);
        cudaMemcpyAsync(T.h[l + 1], T.h[l], sizeof(float) * (size_t)n * kH, cudaMemcpyDeviceToDevice, st);
        launch_node_update_tc(n, T.h[l + 1], T.a[l], L.d_w, o.U[l], o.Ub[l], L.d_err, st);
    }
    float *h3 = T.h[kLayers];
    launch_node_proj_tc(n, h3, L.d_w, o.Po, o.Pob, o.Qo, T.po, T.qo, L.d_err, st);
    edge_kernel<VT, true><<<wrows, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y, blk,
                                                 e.cutoff, T.po, T.qo, L.d_w, o.Ro, o.wo, o.wob, nullptr, L.d_cval,
                                                 L.d_craw);
    diag_out_kernel<<<wrows, 256, 0, st>>>(n, h3, L.d_w, o.wd, o.wdb, L.d_jii, e.d_rowptr, L.d_cval, L.d_crawd);
    // loss: R = R0 - J C Z
    capply_kernel<<<wrows, 256, 0, st>>>(n, k, e.d_rowptr, e.d_col, L.d_cval, T.Z, T.T1);
    jmul_kernel<VT><<<wrows, 256, 0, st>>>(n, k, h, e.d_rowptr, e.d_col, val, T.dvec, T.T1, T.T2, false, 1.0);
    sub_sq_kernel<<<kSubCTAs, 256, 0, st>>>(nk, T.R0, T.T2, T.T1, T.dpart + kSubCTAs); // T1 = R
    // the step follows |R|^2 / |R0|^2: dR = 2 R / |R0|^2; Gm = -J^T dR (into T2)
    scale_by_sum_kernel<<<kSubCTAs, 256, 0, st>>>(nk, 2.0, T.dpart, kSubCTAs, T.T1);
    jmul_kernel<VT><<<wrows, 256, 0, st>>>(n, k, h, e.d_rowptr, e.d_col, val, T.dvec, T.T1, T.T2, true, -1.0);
    const double *Gm = T.T2;
    cudaMemsetAsync(T.g, 0, sizeof(float) * T.nw, st);
    // output layer
    dc_kernel<VT><<<wrows, 256, 0, st>>>(n, k, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, Gm, T.Z, T.dcraw,
                                          T.dcrawd);
    oedge_fwd_kernel<VT><<<kEdgeCTAs, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y, blk,
                                                    e.cutoff, T.po, T.qo, L.d_w, o.Ro, o.wo, T.dcraw, T.dY0, T.epart);
    part_reduce_kernel<<<(kH * kEF + 255) / 256, 256, 0, st>>>(kEdgeWarps, kH * kEF + kH + 1, T.epart, T.g, o.Ro);
    // (the reduce above covers Ro, then wo and wob, which follow Ro in the flat layout)
    oedge_rev_kernel<VT><<<kEdgeCTAs, 256, 0, st>>>(n, k, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y,
                                                    blk, e.cutoff, T.po, T.qo, L.d_w, o.Ro, o.wo, Gm, T.Z, T.dY1);
    dout_w_kernel<<<kH + 1, 256, 0, st>>>(n, T.dcrawd, h3, T.g, o.wd, o.wdb);
    // dh3 = dcrawd w_d + [dpo, dqo] [Po; Qo]; [dPo; dQo] = sum dY (x) h3; dbPo
    cudaMemsetAsync(T.dh, 0, sizeof(float) * (size_t)n * kH, st);
    dout_h_kernel<<<nt, 256, 0, st>>>(n, T.dcrawd, L.d_w, o.wd, T.dh);
    transpose_pq_kernel<<<32, 256, 0, st>>>(L.d_w, o.Po, o.Qo, T.wt_pq);
    const unsigned ntile = (unsigned)((n + 127) / 128);
    tc_dx_kernel<128, 64><<<ntile, 128, 48 * 1024, st>>>(n, T.dY0, T.dY1, T.wt_pq, T.dh, nullptr, true, false,
                                                          L.d_err);
    tc_wgrad_kernel<64><<<kWgradCTAs, 128, 48 * 1024, st>>>(n, T.dY0, T.dY1, h3, nullptr, T.wpart, L.d_err);
    wgrad_reduce_kernel<<<(128 * 64 + 255) / 256, 256, 0, st>>>(kWgradCTAs, 64, T.wpart, T.g, o.Po, o.Qo);
    colsum_kernel<<<kH, 256, 0, st>>>(n, T.dY0, T.g, o.Pob);
    // message-passing rounds, last to first; T.dh holds dh_{l+1}
    for (int l = kLayers - 1; l >= 0; --l) {
        const long nh = (long)n * kH;
        relu_mask_kernel<<<nt, 256, 0, st>>>(nh, T.dh, T.h[l + 1], T.h[l], T.du);
        // [dh; da] += du U (dh_l = dh_{l+1} + ..., da overwritten)
        transpose_u_kernel<<<32, 256, 0, st>>>(L.d_w, o.U[l], T.wt_u);
        // 32 KB of operands; 64 KB requested so that at most three CTAs (3 x 128
        // tensor-memory columns) share an SM and no allocation waits
        tc_dx_kernel<64, 128><<<ntile, 128, 64 * 1024, st>>>(n, T.du, nullptr, T.wt_u, T.dh, T.da, true, false,
                                                              L.d_err);
        tc_wgrad_kernel<128><<<kWgradCTAs, 128, 64 * 1024, st>>>(n, T.du, nullptr, T.h[l], T.a[l], T.wpart, L.d_err);
        wgrad_reduce_kernel<<<(128 * 128 + 255) / 256, 256, 0, st>>>(kWgradCTAs, 128, T.wpart, T.g, o.U[l], -1);
        colsum_kernel<<<kH, 256, 0, st>>>(n, T.du, T.g, o.Ub[l]);
        // the message edges: dph (forward direction) and dqh (reverse)
        ledge_fwd_kernel<VT><<<kEdgeCTAs, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y,
                                                        blk, e.cutoff, T.ph[l], T.qh[l], L.d_w, o.R[l], T.da, T.dY0,
                                                        T.epart);
        part_reduce_kernel<<<(kH * kEF + 255) / 256, 256, 0, st>>>(kEdgeWarps, kH * kEF, T.epart, T.g, o.R[l]);
        ledge_rev_kernel<VT><<<kEdgeCTAs, 256, 0, st>>>(n, h, e.d_rowptr, e.d_col, val, T.dvec, L.d_jii, x, e.d_y,
                                                        blk, e.cutoff, T.ph[l], T.qh[l], L.d_w, o.R[l], T.da, T.dY1);
        // dh_l += [dph, dqh] [P; Q]; [dP; dQ] = sum [dph; dqh] (x) h_l; dbP
        transpose_pq_kernel<<<32, 256, 0, st>>>(L.d_w, o.P[l], o.Q[l], T.wt_pq);
        tc_dx_kernel<128, 64><<<ntile, 128, 48 * 1024, st>>>(n, T.dY0, T.dY1, T.wt_pq, T.dh, nullptr, true, false,
                                                              L.d_err);
        tc_wgrad_kernel<64><<<kWgradCTAs, 128, 48 * 1024, st>>>(n, T.dY0, T.dY1, T.h[l], nullptr, T.wpart, L.d_err);
        wgrad_reduce_kernel<<<(128 * 64 + 255) / 256, 256, 0, st>>>(kWgradCTAs, 64, T.wpart, T.g, o.P[l], o.Q[l]);
        colsum_kernel<<<kH, 256, 0, st>>>(n, T.dY0, T.g, o.Pb[l]);
    }
    din_kernel<<<kH, 256, 0, st>>>(n, T.dh, T.h[0], L.d_nf, T.g, o.in_w, o.in_b);
    e.launches += 40 + 16 * kLayers;
    // loss readback and the optional gradient copy
    std::vector<double> lp(2 * kSubCTAs); // partials of ||R0||^2 (B alone) and ||R||^2 (B + C)
    cudaMemcpyAsync(lp.data(), T.dpart, sizeof(double) * 2 * kSubCTAs, cudaMemcpyDeviceToHost, st);
    if (grad) cudaMemcpyAsync(grad, T.g, sizeof(float) * T.nw, cudaMemcpyDeviceToHost, st);
    if (apply) {
        T.steps++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, (float)T.steps), c2 = 1.0f - std::pow(b2, (float)T.steps);
        norm_kernel<<<1, 1024, 0, st>>>(T.nw, T.g, T.gnorm);
        adam_kernel<<<(unsigned)((T.nw + 255) / 256), 256, 0, st>>>(T.nw, T.W, T.M, T.V, T.g, T.gnorm, 1.0f,
                                                                    (float)lr, b1, b2, 1e-8f, c1, c2, L.d_w);
        L.raw_valid = false;
    }
    if (int rc = e.sync_check("learned training step")) return rc;
    int terr = 0;
    cudaMemcpy(&terr, L.d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (terr) {
        e.err = "learned training: a tensor-core product did not complete";
        return SDDDST_ERR_CUDA;
    }
    if (loss) {
        double s0 = 0.0, s1 = 0.0;
        for (int b = 0; b < kSubCTAs; ++b) {
            s0 += lp[b];
            s1 += lp[kSubCTAs + b];
        }
        loss[0] = s0 / (double)nk;
        loss[1] = s1 / (double)nk;
    }
    return 0;
}

int learned_train_step(Engine &e, double h, int k, double lr, unsigned long long seed, bool apply, double *loss,
                       float *grad)
{
    if (!TR(e)) {
        e.err = "learned training: not started (sdddst_learned_train_init)";
        return SDDDST_ERR_INVALID;
    }
    if (k < 1 || k > kMaxProbes) {
        e.err = "learned training: 1 to 8 probes";
        return SDDDST_ERR_INVALID;
    }
    if (e.valf) return train_step_impl<float>(e, e.d_valf, h, k, lr, seed, apply, loss, grad);
    return train_step_impl<double>(e, e.d_val, h, k, lr, seed, apply, loss, grad);
}

// the FP32 master weights (host, count floats)
int learned_train_weights(Engine &e, float *W, long count)
{
    Train *T = TR(e);
    if (!T || count != T->nw) {
        e.err = "learned training: not started or wrong count";
        return SDDDST_ERR_INVALID;
    }
    cudaMemcpyAsync(W, T->W, sizeof(float) * count, cudaMemcpyDeviceToHost, e.st);
    return e.sync_check("learned weights");
}

} // namespace sd
