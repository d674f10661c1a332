// Linear solve of the chord-Newton system J(h) x = g (the UMFPACK
// symbolic + numeric + solve sequence of the reference,
// src/simulation.cpp:386-396), plus the small vector kernels of the step.
//
// J(h) = I + diag((1 + d)/2) h G is applied matrix-free from the CSR of G
// (warp per row).  The solver is restarted GMRES with classical Gram-Schmidt
// and one re-orthogonalisation pass (CGS2), FP64 throughout, optionally right
// preconditioned by diag(J)^-1.  The (m+1) x m Hessenberg matrix and its
// Givens rotations live on the host; each iteration moves one packed vector
// of 2m+3 doubles device-to-host.  All reductions are two-stage with a fixed
// grid, so results are bit-reproducible run to run.
#include "engine.h"
#include "common.cuh"

#include <cooperative_groups.h>

#include <cmath>
#include <vector>

namespace sd {

// y = J v  (warp per row; G values FP64 or FP32, arithmetic FP64)
// hrow (optional): per-row step size, for block-diagonal batches of systems
template <typename VT>
__global__ void spmv_j_kernel(int n, double h, const double *__restrict__ hrow, const int *__restrict__ rowptr,
                              const int *__restrict__ col, const VT *__restrict__ val,
                              const double *__restrict__ dvec, const double *__restrict__ v, double *__restrict__ y)
{
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const int s = rowptr[row], e = rowptr[row + 1];
    double acc = 0.0;
    for (int q = s + lane; q < e; q += 32) acc += (double)val[q] * v[col[q]];
    acc = warp_sum(acc);
    const double hh = hrow ? hrow[row] : h;
    if (lane == 0) y[row] = v[row] + (1.0 + dvec[row]) * 0.5 * hh * acc;
}

// The same product with the off-diagonal gathers taken from a copy of v in
// the cell-sorted order (vs[k] = v[sorted[k]]): a row's neighbours then lie in
// nine contiguous runs of vs instead of random sectors of v.
template <typename VT, typename IT>
__global__ void spmv_js_kernel(int n, double h, const double *__restrict__ hrow, const int *__restrict__ rowptr,
                               const IT *__restrict__ col_s, const VT *__restrict__ val,
                               const double *__restrict__ dvec, const double *__restrict__ v,
                               const double *__restrict__ vs, double *__restrict__ y)
{
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const int s = rowptr[row], e = rowptr[row + 1];
    double acc = lane == 0 ? (double)val[s] * v[row] : 0.0; // diagonal slot
    for (int q = s + 1 + lane; q < e; q += 32) acc += (double)val[q] * vs[col_s[q]];
    acc = warp_sum(acc);
    const double hh = hrow ? hrow[row] : h;
    if (lane == 0) y[row] = v[row] + (1.0 + dvec[row]) * 0.5 * hh * acc;
}

// The FP32-value, 16-bit-position form with four entries per lane per step:
// 16-byte value loads and 8-byte position loads from the first multiple of
// four in the row on (fewer, wider requests in flight), the unaligned head
// and the tail entry by entry.
__global__ void spmv_js4_kernel(int n, double h, const double *__restrict__ hrow, const int *__restrict__ rowptr,
                                const unsigned short *__restrict__ col_s, const float *__restrict__ val,
                                const double *__restrict__ dvec, const double *__restrict__ v,
                                const double *__restrict__ vs, double *__restrict__ y)
{
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const int s = rowptr[row], e = rowptr[row + 1];
    double acc = lane == 0 ? (double)val[s] * v[row] : 0.0; // diagonal slot
    const int q0 = s + 1;
    const int qa = min(e, (q0 + 3) & ~3);
    if (q0 + lane < qa) acc += (double)val[q0 + lane] * vs[col_s[q0 + lane]];
    for (int q = qa + 4 * lane; q + 3 < e; q += 128) {
        const float4 w = *reinterpret_cast<const float4 *>(val + q);
        const uint2 c = *reinterpret_cast<const uint2 *>(col_s + q);
        acc += (double)w.x * vs[c.x & 0xffffu];
        acc += (double)w.y * vs[c.x >> 16];
        acc += (double)w.z * vs[c.y & 0xffffu];
        acc += (double)w.w * vs[c.y >> 16];
    }
    const int qt = qa + ((e - qa) & ~3);
    if (qt + lane < e) acc += (double)val[qt + lane] * vs[col_s[qt + lane]];
    acc = warp_sum(acc);
    const double hh = hrow ? hrow[row] : h;
    if (lane == 0) y[row] = v[row] + (1.0 + dvec[row]) * 0.5 * hh * acc;
}

__global__ void gather_sorted_kernel(int n, const int *__restrict__ sorted, const double *__restrict__ v,
                                     double *__restrict__ vs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) vs[k] = v[sorted[k]];
}

// diag(J)_i = 1 + (1 + d_i)/2 h G_ii
__global__ void jdiag_inv_kernel(int n, double h, const double *__restrict__ hrow, const double *__restrict__ gdiag,
                                 const double *__restrict__ dvec, double *__restrict__ dinv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dinv[i] = 1.0 / (1.0 + (1.0 + dvec[i]) * 0.5 * (hrow ? hrow[i] : h) * gdiag[i]);
}

__global__ void mul_kernel(int n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] * b[i];
}

__global__ void scale_kernel(int n, double s, const double *__restrict__ a, double *__restrict__ c)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] * s;
}

__global__ void add_kernel(int n, const double *__restrict__ a, double *__restrict__ x)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += a[i];
}

__global__ void sub_kernel(int n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] - b[i];
}

// partials[blk * kk + k] = sum over the block's slice of V[k][i] w[i]
__global__ void multi_dot_partial_kernel(int n, int kk, const double *__restrict__ V, size_t ldv,
                                         const double *__restrict__ w, double *__restrict__ partials)
{
    __shared__ double red[32];
    const int nb = gridDim.x;
    const int chunk = (n + nb - 1) / nb;
    const int s = blockIdx.x * chunk;
    const int e = min(n, s + chunk);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = 0; k < kk; ++k) {
        const double *vk = V + (size_t)k * ldv;
        double acc = 0.0;
        for (int i = s + threadIdx.x; i < e; i += blockDim.x) acc += vk[i] * w[i];
        acc = warp_sum(acc);
        if (lane == 0) red[wid] = acc;
        __syncthreads();
        if (wid == 0) {
            double t = lane < nw ? red[lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) partials[(size_t)blockIdx.x * kk + k] = t;
        }
        __syncthreads();
    }
}

__global__ void multi_dot_final_kernel(int nb, int kk, const double *__restrict__ partials, double *__restrict__ out)
{
    const int k = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __shared__ double red[32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += partials[(size_t)b * kk + k];
    acc = warp_sum(acc);
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    if (wid == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) out[k] = t;
    }
}

// w -= sum_k V[k] c[k]
__global__ void gs_update_kernel(int n, int kk, const double *__restrict__ V, size_t ldv,
                                 const double *__restrict__ c, double *__restrict__ w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = w[i];
    for (int k = 0; k < kk; ++k) acc -= V[(size_t)k * ldv + i] * c[k];
    w[i] = acc;
}

// x += sum_k V[k] y[k]  (optionally times dinv)
__global__ void combine_kernel(int n, int kk, const double *__restrict__ V, size_t ldv, const double *__restrict__ y,
                               const double *__restrict__ dinv, double *__restrict__ x)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (int k = 0; k < kk; ++k) acc += V[(size_t)k * ldv + i] * y[k];
    if (dinv) acc *= dinv[i];
    x[i] += acc;
}

// g_i = x_new - (1+d)/2 h v_new - x_old - (1-d)/2 h v_old (simulation.cpp:189-192)
__global__ void residual_g_kernel(int n, double h0, const double *__restrict__ hrow, const double *__restrict__ xn,
                                  const double *__restrict__ xo, const double *__restrict__ csp,
                                  const double *__restrict__ isp, const double *__restrict__ dvec,
                                  double *__restrict__ g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = hrow ? hrow[i] : h0;
    const double d = dvec[i];
    const double a = __dmul_rn(__dmul_rn(__dmul_rn(__dadd_rn(1.0, d), 0.5), h), csp[i]);
    const double c = __dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(1.0, d), 0.5), h), isp[i]);
    g[i] = __dsub_rn(__dsub_rn(__dsub_rn(xn[i], a), xo[i]), c);
}

// x_new[j] -= x[j] (simulation.cpp:78-81)
__global__ void update_kernel(int n, double *__restrict__ xn, const double *__restrict__ sol)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xn[i] -= sol[i];
}

// ---- generic reductions: op 0 sum a^2, 1 sum |a|, 2 sum b (a - c),
//      3 max over i of (|a - c| > 0 ? (a - c)^2 / b : 0), 4 sum a b
template <int OP>
__device__ __forceinline__ double red_term(int i, const double *a, const double *b, const double *c)
{
    if (OP == 0) return a[i] * a[i];
    if (OP == 1) return fabs(a[i]);
    if (OP == 2) return b[i] * (a[i] - c[i]);
    if (OP == 3) {
        double e = fabs(a[i] - c[i]);
        return e > 0.0 ? __ddiv_rn(__dmul_rn(e, e), b[i]) : 0.0; // precision_handler.cpp:94
    }
    return a[i] * b[i];
}

template <int OP>
__global__ void reduce_partial_kernel(int n, const double *__restrict__ a, const double *__restrict__ b,
                                      const double *__restrict__ c, double *__restrict__ partials)
{
    __shared__ double red[32];
    const int nb = gridDim.x;
    const int chunk = (n + nb - 1) / nb;
    const int s = blockIdx.x * chunk, e = min(n, s + chunk);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double acc = 0.0;
    for (int i = s + threadIdx.x; i < e; i += blockDim.x) {
        double t = red_term<OP>(i, a, b, c);
        acc = OP == 3 ? fmax(acc, t) : acc + t;
    }
    acc = OP == 3 ? warp_max(acc) : warp_sum(acc);
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    if (wid == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = OP == 3 ? warp_max(t) : warp_sum(t);
        if (lane == 0) partials[blockIdx.x] = t;
    }
}

template <int OP>
__global__ void reduce_final_kernel(int nb, const double *__restrict__ partials, double *__restrict__ out)
{
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) acc = OP == 3 ? fmax(acc, partials[k]) : acc + partials[k];
    acc = OP == 3 ? warp_max(acc) : warp_sum(acc);
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    if (wid == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = OP == 3 ? warp_max(t) : warp_sum(t);
        if (lane == 0) *out = t;
    }
}

template <int OP>
static void launch_reduce(Engine &e, int n, const double *a, const double *b, const double *c, double *dst)
{
    reduce_partial_kernel<OP><<<e.red_blocks, 256, 0, e.st>>>(n, a, b, c, e.d_partials);
    reduce_final_kernel<OP><<<1, 256, 0, e.st>>>(e.red_blocks, e.d_partials, dst);
    e.launches += 2;
}

// Reduction with its result copied to the host (synchronises the stream).
int reduce_sum(Engine &e, const double *a, const double *b, int n, int op, double *out)
{
    switch (op) {
    case 0: launch_reduce<0>(e, n, a, nullptr, nullptr, e.d_scal); break;
    case 1: launch_reduce<1>(e, n, a, nullptr, nullptr, e.d_scal); break;
    case 4: launch_reduce<4>(e, n, a, b, nullptr, e.d_scal); break;
    default: return SDDDST_ERR_INVALID;
    }
    cudaMemcpyAsync(e.h_scal, e.d_scal, sizeof(double), cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("reduce")) return rc;
    *out = e.h_scal[0];
    return 0;
}

int Engine::sum_sq(const double *v, double *out) { return reduce_sum(*this, v, nullptr, n, 0, out); }
int Engine::sum_abs(const double *v, double *out) { return reduce_sum(*this, v, nullptr, n, 1, out); }

int Engine::strain_inc(const double *xo, const double *xn, double *out)
{
    launch_reduce<2>(*this, n, xn, d_b, xo, d_scal);
    cudaMemcpyAsync(h_scal, d_scal, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (int rc = sync_check("strain")) return rc;
    *out = h_scal[0];
    return 0;
}

void launch_stage_scalars(Engine &e)
{
    launch_reduce<0>(e, e.n, e.d_v0, nullptr, nullptr, e.d_scal);
    launch_reduce<0>(e, e.n, e.d_v0b, nullptr, nullptr, e.d_scal + 1);
    launch_reduce<3>(e, e.n, e.d_xb, e.d_tol, e.d_x2, e.d_scal + 2);
}

__global__ void fill_kernel(int n, double *__restrict__ p, double v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

void launch_fill(Engine &e, double *p, double v)
{
    fill_kernel<<<(e.n + 255) / 256, 256, 0, e.st>>>(e.n, p, v);
    e.launches++;
}

// sum |v| and sum v^2 in one copy to the host
int Engine::abs_and_sq(const double *v, double *sa, double *sq)
{
    launch_reduce<1>(*this, n, v, nullptr, nullptr, d_scal + 3);
    launch_reduce<0>(*this, n, v, nullptr, nullptr, d_scal + 4);
    cudaMemcpyAsync(h_scal, d_scal + 3, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (int rc = sync_check("speed sums")) return rc;
    *sa = h_scal[0];
    *sq = h_scal[1];
    return 0;
}

// |v0|^2, |v0b|^2 and the error ratio of the step, one copy to the host
int Engine::stage_scalars(double *vs1, double *vs2, double *ratio)
{
    launch_reduce<0>(*this, n, d_v0, nullptr, nullptr, d_scal);
    launch_reduce<0>(*this, n, d_v0b, nullptr, nullptr, d_scal + 1);
    launch_reduce<3>(*this, n, d_xb, d_tol, d_x2, d_scal + 2);
    cudaMemcpyAsync(h_scal, d_scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (int rc = sync_check("step scalars")) return rc;
    *vs1 = h_scal[0];
    *vs2 = h_scal[1];
    *ratio = h_scal[2];
    return 0;
}

int Engine::max_ratio(double *out)
{
    launch_reduce<3>(*this, n, d_xb, d_tol, d_x2, d_scal);
    cudaMemcpyAsync(h_scal, d_scal, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (int rc = sync_check("error ratio")) return rc;
    *out = h_scal[0];
    return 0;
}

void launch_spmv_J(Engine &e, double h, const double *dvec, const double *v, double *y, cudaStream_t st)
{
    const int wpb = 8;
    e.launches++;
    if (e.col_s_valid) {
        e.launches++;
        gather_sorted_kernel<<<(e.n + 255) / 256, 256, 0, st>>>(e.n, e.spmv_sorted, v, e.d_vsort);
        const unsigned nb = (unsigned)((e.n + wpb - 1) / wpb);
        if (e.col_s16_valid) { // 16-bit positions: 2 bytes less per entry
            if (e.valf)
                spmv_js4_kernel<<<nb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr, e.d_col_s16, e.d_valf, dvec, v,
                                                         e.d_vsort, y);
            else
                spmv_js_kernel<double, unsigned short><<<nb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr,
                                                                                 e.d_col_s16, e.d_val, dvec, v,
                                                                                 e.d_vsort, y);
        } else if (e.valf) {
            spmv_js_kernel<float, int><<<nb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr, e.d_col_s, e.d_valf,
                                                                dvec, v, e.d_vsort, y);
        } else {
            spmv_js_kernel<double, int><<<nb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr, e.d_col_s, e.d_val,
                                                                 dvec, v, e.d_vsort, y);
        }
        return;
    }
    if (e.valf)
        spmv_j_kernel<float><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr, e.d_col,
                                                                         e.d_valf, dvec, v, y);
    else
        spmv_j_kernel<double><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(e.n, h, e.d_hrow, e.d_rowptr, e.d_col,
                                                                          e.d_val, dvec, v, y);
}

void launch_residual_g(const Engine &e, double h, const double *xn, const double *xo, const double *csp,
                       const double *isp, const double *dvec, double *g, cudaStream_t st)
{
    residual_g_kernel<<<(e.n + 255) / 256, 256, 0, st>>>(e.n, h, e.d_hrow, xn, xo, csp, isp, dvec, g);
}

void launch_axpy_update(const Engine &e, double *xn, const double *sol, cudaStream_t st)
{
    update_kernel<<<(e.n + 255) / 256, 256, 0, st>>>(e.n, xn, sol);
}

// ---- fused Gram-Schmidt passes: one kernel per pass, each ending in a
// deterministic last-block reduction of the per-block partials.
//   OP 0: out[k] = V[k] . w                       (k < kk)
//   OP 1: w -= V c;  out[k] = V[k] . w            (classical GS, second pass)
//   OP 2: w -= V c;  out[0] = w . w
//   OP 3: out[0] = w . w
template <int OP>
__global__ void __launch_bounds__(256) gs_fused_kernel(int n, int kk, const double *__restrict__ V, size_t ldv,
                                                       double *__restrict__ w, const double *__restrict__ c,
                                                       double *__restrict__ out, double *__restrict__ partials,
                                                       unsigned int *__restrict__ counter)
{
    constexpr int KM = 32;
    __shared__ double cs[KM];
    __shared__ double red[8][KM + 1];
    __shared__ bool last;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if ((OP == 1 || OP == 2) && tid < kk) cs[tid] = c[tid];
    __syncthreads();
    double acc[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) acc[k] = 0.0;
    const int nb = gridDim.x;
    const int chunk = (n + nb - 1) / nb;
    const int s0 = blockIdx.x * chunk, e0 = min(n, s0 + chunk);
    for (int i = s0 + tid; i < e0; i += blockDim.x) {
        double wi = w[i];
        if (OP == 1 || OP == 2) {
            double u = 0.0;
            for (int k = 0; k < kk; ++k) u += V[(size_t)k * ldv + i] * cs[k];
            wi -= u;
            w[i] = wi;
        }
        if (OP == 0 || OP == 1) {
#pragma unroll
            for (int k = 0; k < KM; ++k)
                if (k < kk) acc[k] += V[(size_t)k * ldv + i] * wi;
        } else {
            acc[0] += wi * wi;
        }
    }
    const int nout = (OP == 0 || OP == 1) ? kk : 1;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        if (k < nout) {
            double v = warp_sum(acc[k]);
            if (lane == 0) red[wid][k] = v;
        }
    }
    __syncthreads();
    if (tid < nout) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q][tid];
        partials[(size_t)blockIdx.x * KM + tid] = t;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (tid < nout) {
        double t = 0.0;
        for (int b = 0; b < nb; ++b) t += partials[(size_t)b * KM + tid];
        out[tid] = t;
    }
    if (tid == 0) *counter = 0u;
}

// One whole Gram-Schmidt step of GMRES in a single cooperative launch (one
// CTA per SM, grid-wide barriers between the passes): c1 = V^T w, w -= V c1,
// c2 = V^T w with |w|^2, w -= V c2, nrm2 = |w|^2 before - |c2|^2,
// V_{k+1} = w / sqrt(nrm2).  Each CTA owns a contiguous range of the
// vectors; the per-CTA partial sums are reduced by every CTA in the same
// fixed order (identical results, no further barrier).  rec receives c1 at
// [0, m1), c2 at [m1, 2 m1) and nrm2 at [2 m1], the layout of the three
// separate passes.
//
// Per-CTA partials of V^T w (entries 0 .. kk-1) and, with with_norm, of
// |w|^2 as entry kk (kk <= 31).
__device__ __forceinline__ void gs_block_dots(int kk, const double *__restrict__ V, size_t ldv, const double *w,
                                              int s0, int e0, double (*red)[33], double *__restrict__ part,
                                              bool with_norm)
{
    constexpr int KM = 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double acc[KM];
    double accn = 0.0;
#pragma unroll
    for (int k = 0; k < KM; ++k) acc[k] = 0.0;
    for (int i = s0 + tid; i < e0; i += blockDim.x) {
        const double wi = w[i];
        if (with_norm) accn += wi * wi;
#pragma unroll
        for (int k = 0; k < KM; ++k)
            if (k < kk) acc[k] += V[(size_t)k * ldv + i] * wi;
    }
    const int nout = with_norm ? kk + 1 : kk;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        if (k < nout) {
            const double v = warp_sum(with_norm && k == kk ? accn : acc[k]);
            if (lane == 0) red[wid][k] = v;
        }
    }
    __syncthreads();
    if (tid < nout) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q][tid];
        part[tid] = t;
    }
    __threadfence();
}

// sums_s[k] = sum over the nb per-CTA partials of entry k, k < cnt: one warp
// per entry, lane-strided partial sums then a butterfly, lane 0's result
// kept (a fixed order, so every CTA computes the same values).  A serial sum
// over the partials would put nb dependent L2 round trips on the critical
// path of every pass.
__device__ __forceinline__ void gs_sum_partials(const double *__restrict__ part, int nb, int cnt, double *sums_s)
{
    constexpr int KM = 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = wid; k < cnt; k += nw) {
        double t = 0.0;
        for (int b = lane; b < nb; b += 32) t += part[(size_t)b * KM + k];
        t = warp_sum(t);
        if (lane == 0) sums_s[k] = t;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) gs_iter_kernel(int n, int kk, const double *__restrict__ V, size_t ldv,
                                                      double *__restrict__ w, double *__restrict__ rec, int m1,
                                                      double *__restrict__ partials, double *__restrict__ vnext)
{
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    constexpr int KM = 32;
    __shared__ double cs[KM];
    __shared__ double red[8][KM + 1];
    const int tid = threadIdx.x, nb = gridDim.x;
    const int chunk = (n + nb - 1) / nb;
    const int s0 = blockIdx.x * chunk, e0 = min(n, s0 + chunk);
    // the second pass also sums |w1|^2; with V orthonormal the final norm is
    // |w1 - V c2|^2 = |w1|^2 - |c2|^2, and c2 (the re-orthogonalisation) is
    // tiny against w1, so the difference loses nothing: two grid barriers
    double nrm2 = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        double *part = partials + ((size_t)pass * nb) * KM;
        gs_block_dots(kk, V, ldv, w, s0, e0, red, part + (size_t)blockIdx.x * KM, pass == 1);
        grid.sync();
        gs_sum_partials(part, nb, pass == 1 ? kk + 1 : kk, cs);
        if (blockIdx.x == 0 && tid < kk) rec[pass * m1 + tid] = cs[tid];
        if (pass == 1) {
            double c2 = 0.0;
            for (int k = 0; k < kk; ++k) c2 += cs[k] * cs[k];
            nrm2 = fmax(cs[kk] - c2, 0.0);
        }
        for (int i = s0 + tid; i < e0; i += blockDim.x) {
            double u = 0.0;
            for (int k = 0; k < kk; ++k) u += V[(size_t)k * ldv + i] * cs[k];
            const double wn = w[i] - u;
            w[i] = wn;
            if (pass == 1) vnext[i] = nrm2 > 0.0 ? wn * rsqrt(nrm2) : 0.0;
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && tid == 0) rec[2 * m1] = nrm2;
}

// The cooperative Gram-Schmidt step runs when the device supports cooperative
// launches and `blocks` CTAs of it fit on the device at once.
bool gs_coop_supported(int device, int blocks)
{
    int coop = 0, sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return false;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return false;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gs_iter_kernel, 256, 0) != cudaSuccess) return false;
    return blocks <= per_sm * sms;
}

// V_{j+1} = w / sqrt(nrm2) (zero vector on breakdown)
__global__ void normalize_kernel(int n, const double *__restrict__ w, const double *__restrict__ nrm2,
                                 double *__restrict__ v)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = *nrm2;
    v[i] = s > 0.0 ? w[i] * rsqrt(s) : 0.0;
}

// Restarted GMRES(m) on J(h) x = rhs, x0 = 0, right preconditioned
// (precond 0: none, 1: diagonal, 2: cluster blocks, 3: sparse LU factors, 4: cluster
// blocks plus the learned correction).  Iterations run without
// host synchronisation; every `chk` iterations the Hessenberg columns come
// back in one copy, the host applies the Givens rotations and tests
// convergence (so at most chk-1 iterations past convergence are computed).
// Returns 0 on reaching e.prm.solver_tol relative residual.
int gmres_solve(Engine &e, double h, const double *dvec, const double *rhs, double *x, int precond)
{
    const int n = e.n, m = e.restart;
    const size_t ldv = (size_t)n;
    cudaStream_t st = e.st;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const double tol = e.prm.solver_tol > 0 ? e.prm.solver_tol : 1e-13;
    const int max_it = e.prm.max_iters > 0 ? e.prm.max_iters : 1000;
    // convergence is checked on the host after a chunk of iterations: the
    // first chunk is as long as the previous solve of this engine took
    // (consecutive solves of a step need similar counts), later ones 2
    const int first_chk = std::max(2, std::min(m, e.gmres_hint));
    const int chk = 2;
    const int stride = 2 * (m + 1) + 1; // per-iteration record: c1[m+1], c2[m+1], nrm2
    double *V = e.d_V, *w = e.d_w, *z = e.d_z, *r = e.d_r;
    double *dinv = nullptr;
    cudaMemsetAsync(x, 0, sizeof(double) * n, st);
    if (precond == 1) {
        dinv = e.d_y_small; // n doubles reserved for the diagonal
        jdiag_inv_kernel<<<nb, 256, 0, st>>>(n, h, e.d_hrow, e.d_gdiag, dvec, dinv);
        e.launches++;
    }
    auto apply_precond = [&](const double *in, double *out) -> const double * {
        if (precond == 1) {
            mul_kernel<<<nb, 256, 0, st>>>(n, in, dinv, out);
            e.launches++;
            return out;
        }
        if (precond == 2) {
            precond_apply(e, in, out);
            return out;
        }
        if (precond == 3) {
            direct_apply(e, in, out);
            return out;
        }
        if (precond == 4) {
            precond_apply(e, in, out);
            learned_apply_add(e, in, out);
            return out;
        }
        return in;
    };
    // beta0 = ||rhs||
    cudaMemcpyAsync(r, rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    gs_fused_kernel<3><<<e.gs_blocks, 256, 0, st>>>(n, 1, nullptr, ldv, r, nullptr, e.d_scal, e.d_partials,
                                                     e.d_counter);
    e.launches++;
    cudaMemcpyAsync(e.h_scal, e.d_scal, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("gmres start")) return rc;
    double beta0 = std::sqrt(e.h_scal[0]);
    e.last_iters = 0;
    e.last_resid = 0.0;
    if (beta0 == 0.0) return 0;
    if (!std::isfinite(beta0)) {
        e.err = "solve: non-finite right-hand side";
        return SDDDST_ERR_NONFINITE;
    }
    double beta = beta0;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1), yv(m);
    double *hrec = e.h_hrec;
    int total = 0;
    bool converged = false;
    while (!converged) {
        normalize_kernel<<<nb, 256, 0, st>>>(n, r, e.d_scal, V); // d_scal holds ||r||^2
        e.launches++;
        std::fill(gv.begin(), gv.end(), 0.0);
        gv[0] = beta;
        int k = 0;
        int j = 0;
        bool stop = false;
        bool first_chunk = true;
        while (j < m && !stop) {
            const int jend = std::min(m, j + (first_chunk ? first_chk : chk));
            first_chunk = false;
            for (int jj = j; jj < jend; ++jj) {
                const double *src = apply_precond(V + (size_t)jj * ldv, z);
                launch_spmv_J(e, h, dvec, src, w, st);
                double *rec = e.d_hrec + (size_t)jj * stride;
                const int kk = jj + 1;
                if (e.coop_gs) {
                    int a_n = n, a_kk = kk, a_m1 = m + 1;
                    size_t a_ldv = ldv;
                    double *a_V = V, *a_w = w, *a_rec = rec, *a_part = e.d_gs_partials;
                    double *a_next = V + (size_t)(jj + 1) * ldv;
                    void *args[] = {&a_n, &a_kk, &a_V, &a_ldv, &a_w, &a_rec, &a_m1, &a_part, &a_next};
                    if (cudaLaunchCooperativeKernel((const void *)gs_iter_kernel, dim3(e.gs_blocks), dim3(256), args,
                                                    0, st) == cudaSuccess) {
                        e.launches++;
                        continue;
                    }
                    (void)cudaGetLastError(); // not launchable here: the separate passes from now on
                    e.coop_gs = false;
                }
                gs_fused_kernel<0><<<e.gs_blocks, 256, 0, st>>>(n, kk, V, ldv, w, nullptr, rec, e.d_partials,
                                                                 e.d_counter);
                gs_fused_kernel<1><<<e.gs_blocks, 256, 0, st>>>(n, kk, V, ldv, w, rec, rec + (m + 1), e.d_partials,
                                                                 e.d_counter);
                gs_fused_kernel<2><<<e.gs_blocks, 256, 0, st>>>(n, kk, V, ldv, w, rec + (m + 1), rec + 2 * (m + 1),
                                                                 e.d_partials, e.d_counter);
                normalize_kernel<<<nb, 256, 0, st>>>(n, w, rec + 2 * (m + 1), V + (size_t)(jj + 1) * ldv);
                e.launches += 4;
            }
            cudaMemcpyAsync(hrec + (size_t)j * stride, e.d_hrec + (size_t)j * stride,
                            sizeof(double) * stride * (jend - j), cudaMemcpyDeviceToHost, st);
            if (int rc = e.sync_check("gmres iteration")) return rc;
            for (int jj = j; jj < jend && !stop; ++jj) {
                const double *rc = hrec + (size_t)jj * stride;
                const double hn = std::sqrt(std::max(rc[2 * (m + 1)], 0.0));
                for (int i = 0; i <= jj; ++i) H[(size_t)i * m + jj] = rc[i] + rc[(m + 1) + i];
                H[(size_t)(jj + 1) * m + jj] = hn;
                if (!std::isfinite(hn)) {
                    e.err = "solve: non-finite Krylov vector";
                    return SDDDST_ERR_NONFINITE;
                }
                for (int i = 0; i < jj; ++i) {
                    double a = H[(size_t)i * m + jj], b2 = H[(size_t)(i + 1) * m + jj];
                    H[(size_t)i * m + jj] = cs[i] * a + sn[i] * b2;
                    H[(size_t)(i + 1) * m + jj] = -sn[i] * a + cs[i] * b2;
                }
                double a = H[(size_t)jj * m + jj], b2 = H[(size_t)(jj + 1) * m + jj];
                double rr = std::hypot(a, b2);
                cs[jj] = rr > 0 ? a / rr : 1.0;
                sn[jj] = rr > 0 ? b2 / rr : 0.0;
                H[(size_t)jj * m + jj] = rr;
                H[(size_t)(jj + 1) * m + jj] = 0.0;
                gv[jj + 1] = -sn[jj] * gv[jj];
                gv[jj] = cs[jj] * gv[jj];
                ++total;
                k = jj + 1;
                if (std::fabs(gv[jj + 1]) <= tol * beta0 || hn == 0.0) {
                    converged = true;
                    stop = true;
                }
                if (total >= max_it) stop = true;
            }
            j = jend;
        }
        // back substitution and x += M^-1 V y
        for (int i = k - 1; i >= 0; --i) {
            double s = gv[i];
            for (int q = i + 1; q < k; ++q) s -= H[(size_t)i * m + q] * yv[q];
            yv[i] = s / H[(size_t)i * m + i];
        }
        cudaMemcpyAsync(e.d_y_small + n, yv.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st);
        if (precond >= 2) {
            cudaMemsetAsync(r, 0, sizeof(double) * n, st);
            combine_kernel<<<nb, 256, 0, st>>>(n, k, V, ldv, e.d_y_small + n, nullptr, r);
            if (precond == 2) precond_apply(e, r, z);
            else if (precond == 3) direct_apply(e, r, z);
            else {
                precond_apply(e, r, z);
                learned_apply_add(e, r, z);
            }
            add_kernel<<<nb, 256, 0, st>>>(n, z, x);
            e.launches += 2;
        } else {
            combine_kernel<<<nb, 256, 0, st>>>(n, k, V, ldv, e.d_y_small + n, dinv, x);
            e.launches++;
        }
        if (converged || total >= max_it) break;
        // restart from the true residual
        launch_spmv_J(e, h, dvec, x, w, st);
        sub_kernel<<<nb, 256, 0, st>>>(n, rhs, w, r);
        gs_fused_kernel<3><<<e.gs_blocks, 256, 0, st>>>(n, 1, nullptr, ldv, r, nullptr, e.d_scal, e.d_partials,
                                                         e.d_counter);
        e.launches += 2;
        cudaMemcpyAsync(e.h_scal, e.d_scal, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (int rc = e.sync_check("gmres restart")) return rc;
        beta = std::sqrt(e.h_scal[0]);
        if (beta <= tol * beta0) {
            converged = true;
            break;
        }
    }
    e.last_iters = total;
    if (converged && total > 0) e.gmres_hint = total;
    e.solves++;
    e.iterations += total;
    if (!converged) {
        e.err = "solve: GMRES did not reach the residual target";
        return SDDDST_ERR_SOLVER;
    }
    return 0;
}

} // namespace sd
