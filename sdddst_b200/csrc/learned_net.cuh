// The learned preconditioner's network, shared by its inference
// (learned.cu) and its training (learned_train.cu): sizes, the flat BF16
// weight layout (the order of sdddst_b200/learned.py, weight_tensors), the
// engine-side state, and the forward kernels over the CSR of J.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "engine.h"

namespace sd {

// node_gemm_tc.cu: the node products on the tensor cores
void launch_node_proj_tc(int n, const float *h, const __nv_bfloat16 *w, long oP, long oPb, long oQ, float *ph,
                         __nv_bfloat16 *qh, int *err, cudaStream_t st);
void launch_node_update_tc(int n, float *h, const float *a, const __nv_bfloat16 *w, long oU, long oUb, int *err,
                           cudaStream_t st);

namespace ln {

constexpr int kH = 64, kNF = 4, kEF = 5, kLayers = 3;
constexpr float kDegScale = 627.0f, kPosScale = 7.0f;

struct WeightOffsets {
    long in_w, in_b;
    long P[kLayers], Pb[kLayers], Q[kLayers], R[kLayers], U[kLayers], Ub[kLayers];
    long Po, Pob, Qo, Ro, wo, wob, wd, wdb, total;
};

inline WeightOffsets offsets()
{
    WeightOffsets o{};
    long p = 0;
    auto take = [&](long k) {
        const long at = p;
        p += k;
        return at;
    };
    o.in_w = take(kH * kNF);
    o.in_b = take(kH);
    for (int l = 0; l < kLayers; ++l) {
        o.P[l] = take(kH * kH);
        o.Pb[l] = take(kH);
        o.Q[l] = take(kH * kH);
        o.R[l] = take(kH * kEF);
        o.U[l] = take(kH * 2 * kH);
        o.Ub[l] = take(kH);
    }
    o.Po = take(kH * kH);
    o.Pob = take(kH);
    o.Qo = take(kH * kH);
    o.Ro = take(kH * kEF);
    o.wo = take(kH);
    o.wob = take(1);
    o.wd = take(kH);
    o.wdb = take(1);
    o.total = p;
    return o;
}

struct Learned {
    bool has_weights = false;
    bool compact = false;                   // the analytic correction is held in its compact CSR
    int *d_crow = nullptr, *d_ccnt = nullptr, *d_ccol = nullptr;
    float *d_cv = nullptr;
    __nv_bfloat16 *d_w = nullptr;
    WeightOffsets off{};
    float *d_nf = nullptr, *d_h = nullptr, *d_ph = nullptr, *d_agg = nullptr;
    __nv_bfloat16 *d_qh = nullptr;          // Q h in BF16 (the per-edge gather)
    int *d_err = nullptr, *h_err = nullptr; // a tensor-core wait that ran out (device flag, pinned copy)
    double *d_jii = nullptr;
    float *d_cval = nullptr;
    float *d_craw = nullptr, *d_crawd = nullptr; // the network's raw outputs of the last inference
    long cval_cap = 0, ccap = 0;
    long builds = 0, rescales = 0;
    bool raw_valid = false; // d_craw / d_crawd hold the outputs of an inference on the current assembly
    // the pattern those outputs belong to (row pointers, columns), kept across
    // the next assembly so its C can reuse them (learned_remap)
    int *d_rp0 = nullptr, *d_col0 = nullptr;
    float *d_craw0 = nullptr; // remap target
    long col0_cap = 0;
    bool prev_valid = false;
    int remaps = 0;           // assemblies served by remapping since the last inference
    long remap_count = 0;
    void *train = nullptr;  // training state (learned_train.cu)
};

inline Learned *LN(Engine &e) { return static_cast<Learned *>(e.learned); }

__device__ __forceinline__ float bf(const __nv_bfloat16 *w, long i) { return __bfloat162float(w[i]); }
__device__ __forceinline__ float tlogf(float v) { return copysignf(log1pf(fabsf(v)), v); }

namespace { // the kernels: one copy per translation unit

// node features and J_ii; one warp per row
template <typename VT>
__global__ void feat_kernel(int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                            const VT *__restrict__ val, const double *__restrict__ gdiag,
                            const double *__restrict__ dvec, float *__restrict__ nf, double *__restrict__ jii)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double di = (1.0 + dvec[i]) * 0.5 * h;
    double rs = 0.0, cs = 0.0;
    int deg = 0;
    for (int q = rowptr[i] + lane; q < rowptr[i + 1]; q += 32) {
        const int j = col[q];
        if (j == i) continue;
        const double g = (double)val[q];
        rs += fabs(di * g);
        cs += fabs((1.0 + dvec[j]) * 0.5 * h * g);
        ++deg;
    }
    rs = warp_sum(rs);
    cs = warp_sum(cs);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) deg += __shfl_xor_sync(0xffffffffu, deg, o);
    if (lane == 0) {
        const double aii = di * gdiag[i];
        jii[i] = 1.0 + aii;
        nf[4 * i + 0] = tlogf((float)aii);
        nf[4 * i + 1] = tlogf((float)rs);
        nf[4 * i + 2] = tlogf((float)cs);
        nf[4 * i + 3] = (float)deg / kDegScale;
    }
}

__global__ void node_in_kernel(int n, const float *__restrict__ nf, const __nv_bfloat16 *__restrict__ w, long ow,
                               long ob, float *__restrict__ hout)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * kH) return;
    const int i = (int)(idx >> 6), c = (int)(idx & 63);
    float acc = bf(w, ob + c);
#pragma unroll
    for (int f = 0; f < kNF; ++f) acc = fmaf(bf(w, ow + c * kNF + f), nf[4 * i + f], acc);
    hout[idx] = fmaxf(acc, 0.0f);
}

// per-edge pass, one warp per row, 8 rows per block of 256 threads: lane l
// holds channels 2l and 2l + 1 (one 4-byte BF16 pair of qh_j per edge,
// packed FP32 arithmetic); a chunk's 32 edges have their features formed one
// per lane and staged in shared memory, every lane then reads them back
// (two 16-byte broadcast loads per edge).
// kOut = false: agg_i = mean_j relu(ph_i + qh_j + R e_ij);
// kOut = true:  C_ij = (w_o . relu(ph_i + qh_j + R e_ij) + b_o) A_ij / (J_ii J_jj)
template <typename VT, bool kOut>
__global__ void __launch_bounds__(256)
    edge_kernel(int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                const VT *__restrict__ val, const double *__restrict__ dvec, const double *__restrict__ jii,
                const double *__restrict__ x, const double *__restrict__ y, const int *__restrict__ blk,
                double cutoff, const float *__restrict__ ph, const __nv_bfloat16 *__restrict__ qh,
                const __nv_bfloat16 *__restrict__ w, long oR, long owo, long owob, float *__restrict__ agg,
                float *__restrict__ cval, float *__restrict__ craw)
{
    __shared__ __align__(16) float sfeat[8][32][8]; // per warp: e0..e3 | e4, j (bits), -, -
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, wib = (threadIdx.x >> 5) & 7;
    if (i >= n) return;
    const int c0 = 2 * lane;
    float2 rf[kEF];
#pragma unroll
    for (int f = 0; f < kEF; ++f) rf[f] = make_float2(bf(w, oR + c0 * kEF + f), bf(w, oR + (c0 + 1) * kEF + f));
    float2 wo = make_float2(0.0f, 0.0f);
    float bo = 0.0f;
    if (kOut) {
        wo = make_float2(bf(w, owo + c0), bf(w, owo + c0 + 1));
        bo = bf(w, owob);
    }
    const float2 pp = *reinterpret_cast<const float2 *>(ph + (long)i * kH + c0);
    const double di = (1.0 + dvec[i]) * 0.5 * h;
    const double ji = jii[i];
    const double xi = x[i], yi = y[i];
    const int bi = blk[i];
    const float inv_pos = (float)(1.0 / (kPosScale * cutoff));
    float2 s = make_float2(0.0f, 0.0f);
    int cnt = 0;
    float *my = &sfeat[wib][lane][0];
    const int qs = rowptr[i], qe = rowptr[i + 1];
    for (int q0 = qs; q0 < qe; q0 += 32) {
        const int q = q0 + lane;
        int j = -1;
        float e0 = 0.f, e1 = 0.f, e2 = 0.f, e3 = 0.f, e4 = 0.f, sc = 0.f;
        if (q < qe) {
            j = col[q];
            if (j != i) {
                const double g = (double)val[q];
                const double aij = di * g, aji = (1.0 + dvec[j]) * 0.5 * h * g;
                double dx = x[j] - xi, dy = y[j] - yi;
                dx -= rint(dx);
                dy -= rint(dy);
                e0 = tlogf((float)aij);
                e1 = tlogf((float)aji);
                e2 = (float)dx * inv_pos;
                e3 = (float)dy * inv_pos;
                e4 = blk[j] == bi ? 1.0f : 0.0f;
                sc = (float)(aij / (ji * jii[j]));
            } else {
                j = -2; // the diagonal slot is no edge (its C value comes from the diagonal output)
            }
        }
        cnt += __popc(__ballot_sync(0xffffffffu, j >= 0));
        *reinterpret_cast<float4 *>(my) = make_float4(e0, e1, e2, e3);
        *reinterpret_cast<float4 *>(my + 4) = make_float4(e4, __int_as_float(j), 0.0f, 0.0f);
        __syncwarp();
        // the chunk's 32 edges unrolled: independent gathers of qh_j; the
        // output pass leaves lane t's two-channel partial of edge t in v[t]
        float v[32];
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const float4 fa = *reinterpret_cast<const float4 *>(&sfeat[wib][t][0]);
            const float4 fb = *reinterpret_cast<const float4 *>(&sfeat[wib][t][4]);
            const int jt = __float_as_int(fb.y);
            float2 a = make_float2(0.0f, 0.0f);
            if (jt >= 0) {
                const __nv_bfloat162 qv = *reinterpret_cast<const __nv_bfloat162 *>(qh + (long)jt * kH + c0);
                a = __fadd2_rn(pp, __bfloat1622float2(qv));
                a = __ffma2_rn(rf[0], make_float2(fa.x, fa.x), a);
                a = __ffma2_rn(rf[1], make_float2(fa.y, fa.y), a);
                a = __ffma2_rn(rf[2], make_float2(fa.z, fa.z), a);
                a = __ffma2_rn(rf[3], make_float2(fa.w, fa.w), a);
                a = __ffma2_rn(rf[4], make_float2(fb.x, fb.x), a);
                a.x = fmaxf(a.x, 0.0f);
                a.y = fmaxf(a.y, 0.0f);
            }
            if (kOut) v[t] = fmaf(wo.x, a.x, wo.y * a.y);
            else s = __fadd2_rn(s, a);
        }
        __syncwarp(); // the next chunk overwrites the staged features
        if (kOut) {
            // reduce-scatter over the warp: afterwards lane l holds the sum
            // over all lanes of v[l] in v[0] (31 shuffles for 32 edges)
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                const bool up = (lane & o) != 0;
#pragma unroll
                for (int k = 0; k < o; ++k) {
                    const float send = up ? v[k] : v[k + o];
                    const float keep = up ? v[k + o] : v[k];
                    v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
            if (j >= 0) {
                const float c = v[0] + bo; // the network's part of c_ij
                cval[q] = (c - (1.0f - e4)) * sc;
                craw[q] = c;
            }
        }
    }
    if (!kOut) {
        const float inv = 1.0f / (float)max(cnt, 1);
        *reinterpret_cast<float2 *>(agg + (long)i * kH + c0) = make_float2(s.x * inv, s.y * inv);
    }
}

// C_ii = (w_d . h_i + b_d) / J_ii into each row's diagonal slot (slot 0)
__global__ void diag_out_kernel(int n, const float *__restrict__ hin, const __nv_bfloat16 *__restrict__ w, long owd,
                                long owdb, const double *__restrict__ jii, const int *__restrict__ rowptr,
                                float *__restrict__ cval, float *__restrict__ crawd)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    float v = bf(w, owd + lane) * hin[(long)i * kH + lane] + bf(w, owd + lane + 32) * hin[(long)i * kH + lane + 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) {
        const float c = v + bf(w, owdb);
        cval[rowptr[i]] = (float)(c / jii[i]);
        crawd[i] = c;
    }
}

} // namespace

} // namespace ln

} // namespace sd
