// Device-resident GMRES(m): one whole chord-Newton solve J(h) x = g (the
// UMFPACK factor + solve of the reference, src/simulation.cpp:386-396) in ONE
// cooperative launch, for one system or for two systems that share G.
//
// Stage I (h) and stage II (h/2) of a step start from the same configuration
// and share the Jacobian's unit-step part G (J(h) = I + diag((1+d)/2) h G), so
// their solves run together: every SpMV pass reads G's values and column
// positions once and applies them to both Krylov vectors.  Everything an
// iteration needs stays on the device:
//   P1  z = M^-1 V_j (cluster block-Jacobi), written in the user order and in
//       the cell-sorted order the SpMV gathers from;
//   P2  w = J z (warp per row; CTAs take rows dynamically in cell-sorted
//       order), then, after a barrier, the CTA's partial dots V_k . w over its
//       own static rows;
//   P3  reduced c1, w -= V c1, partial dots V_k . w and |w|^2 (second
//       Gram-Schmidt pass);
//   P4  reduced c2, w -= V c2, V_{j+1} = w / |w| (|w|^2 = |w1|^2 - |c2|^2),
//       the Givens rotation of the new Hessenberg column and the convergence
//       test |g_{j+1}| <= tol beta0;
// with a grid barrier after each phase.  Every CTA owns a contiguous range of
// rows (and of cell-sorted positions) and reduces the per-CTA partial sums in
// the same fixed order, so all CTAs hold identical Hessenberg columns, apply
// identical rotations and take the same decisions; results are bit-identical
// run to run.  At the end of a cycle the small triangular system is solved in
// every CTA, x += M^-1 V y, and a restart (rare) recomputes r = g - J x.
#include "engine.h"
#include "common.cuh"

#include <cooperative_groups.h>

#include <cmath>

namespace sd {

namespace {

constexpr int kThreads = 512;
constexpr int kKM = 32; // restart length bound (m <= 31) and partial-sum stride
constexpr int kStatusSlots = 8; // solves whose statuses one attempt can leave on the device
constexpr int kPasses = 1024;   // ring of SpMV row counters (a pass zeroes the next one)

struct FusedSys {
    double h;
    const double *hrow; // per-row step size (a batch of systems), or null: h
    const double *dvec;
    const double *rhs;
    double *x;
    double *V;          // (m + 1) x n
    double *w, *z, *zs; // n each: A z, M^-1 V_j (user order), the same in the cell-sorted order
    const int *blk_of, *loc, *bstart, *blen, *members, *off;
    const double *binv;
    double *status; // [0] iterations [1] converged [2] |g_k| / beta0 [3] non-finite
};

struct FusedArgs {
    int n, m, max_it;
    double tol;
    const int *rowptr;
    const void *cols;  // cell-sorted column positions (IT), diagonal slot unused
    const void *vals;  // G values (VT), diagonal in each row's first slot
    const int *sorted; // cell-sorted position -> dislocation
    const int2 *srow;  // cell-sorted position -> its row's (start, end) in the CSR
    double *part;      // per-CTA partial sums: [2 passes][2 systems][kKM][grid] (a sum's partials contiguous)
    int *ctr;          // SpMV row counters, one per pass (ring of kPasses)
    FusedSys sys[2];
};

// M^-1 v at dislocation i (its row of its block's inverse)
__device__ __forceinline__ double block_row(const FusedSys &S, int i, const double *__restrict__ v)
{
    const int b = S.blk_of[i];
    const int k = S.blen[b], s = S.bstart[b];
    const double *B = S.binv + S.off[b] + (size_t)S.loc[i] * k;
    double acc = 0.0;
    for (int c = 0; c < k; ++c) acc += B[c] * v[S.members[s + c]];
    return acc;
}

// One warp: the off-diagonal sum of row `row` of G against the cell-sorted
// vectors zs0 (and zs1 when NS == 2); the diagonal slot is added by lane 0.
template <typename VT, typename IT, int NS>
struct RowDot;

// FP32 values, 16-bit cell-sorted positions.  Two forms, measured on the
// N=32768 workload (SpMV phase of a solve, about five passes):
//   one vector (stage III): a lane holds four consecutive entries (16-byte
//   value and 8-byte position loads), two 128-entry chunks per step: 185 us;
//   lanes on consecutive entries (scalar coalesced loads): 209 us;
//   two vectors (stages I+II): 385 us and 345 us -- with two gathers per
//   entry the gathers' spread over cache lines dominates, and consecutive
//   lanes on consecutive entries read neighbouring doubles.
template <>
struct RowDot<float, unsigned short, 1> {
    __device__ __forceinline__ static void run(int s, int e, int lane, const float *__restrict__ val,
                                               const unsigned short *__restrict__ col, const double *__restrict__ a,
                                               const double *__restrict__ b, double &acc0, double &acc1)
    {
        (void)b;
        (void)acc1;
        const int q0 = s + 1;
        const int qa = min(e, (q0 + 3) & ~3);
        if (q0 + lane < qa) acc0 += (double)val[q0 + lane] * a[col[q0 + lane]];
        // both chunks' value and position loads are issued before their gathers
        for (int q = qa + 4 * lane; q + 3 < e; q += 256) {
            const bool two = q + 131 < e;
            const float4 w = *reinterpret_cast<const float4 *>(val + q);
            const uint2 c = *reinterpret_cast<const uint2 *>(col + q);
            float4 w2 = make_float4(0.f, 0.f, 0.f, 0.f);
            uint2 cc = make_uint2(0u, 0u);
            if (two) {
                w2 = *reinterpret_cast<const float4 *>(val + q + 128);
                cc = *reinterpret_cast<const uint2 *>(col + q + 128);
            }
            const double a0 = a[c.x & 0xffffu], a1 = a[c.x >> 16], a2 = a[c.y & 0xffffu], a3 = a[c.y >> 16];
            const double a4 = a[cc.x & 0xffffu], a5 = a[cc.x >> 16], a6 = a[cc.y & 0xffffu],
                         a7 = a[cc.y >> 16]; // position 0 when !two (w2 = 0)
            acc0 += (double)w.x * a0;
            acc0 += (double)w.y * a1;
            acc0 += (double)w.z * a2;
            acc0 += (double)w.w * a3;
            acc0 += (double)w2.x * a4;
            acc0 += (double)w2.y * a5;
            acc0 += (double)w2.z * a6;
            acc0 += (double)w2.w * a7;
        }
        const int qt = qa + ((e - qa) & ~3);
        if (qt + lane < e) acc0 += (double)val[qt + lane] * a[col[qt + lane]];
    }
};

// lanes on consecutive entries, one (kTwo false) or two vectors
template <bool kTwo>
__device__ __forceinline__ void row_dot_coalesced(int s, int e, int lane, const float *__restrict__ val,
                                                  const unsigned short *__restrict__ col,
                                                  const double *__restrict__ a, const double *__restrict__ b,
                                                  double &acc0, double &acc1)
{
    constexpr int kU = 8;
    for (int q = s + 1 + lane; q < e; q += 32 * kU) {
        float w[kU];
        int c[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int qq = q + 32 * u;
            const bool in = qq < e;
            w[u] = in ? val[qq] : 0.0f; // position 0, weight 0 past the row
            c[u] = in ? (int)col[qq] : 0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            acc0 += (double)w[u] * a[c[u]];
            if (kTwo) acc1 += (double)w[u] * b[c[u]];
        }
    }
}

template <>
struct RowDot<float, unsigned short, 2> {
    __device__ __forceinline__ static void run(int s, int e, int lane, const float *__restrict__ val,
                                               const unsigned short *__restrict__ col, const double *__restrict__ a,
                                               const double *__restrict__ b, double &acc0, double &acc1)
    {
        row_dot_coalesced<true>(s, e, lane, val, col, a, b, acc0, acc1);
    }
};

// One active vector inside a kernel built for NS systems: the joint kernel
// (NS = 2) keeps the coalesced form, whose registers it already holds.
template <typename VT, typename IT, int NS>
struct RowDot1 {
    __device__ __forceinline__ static void run(int s, int e, int lane, const VT *__restrict__ val,
                                               const IT *__restrict__ col, const double *__restrict__ a,
                                               double &acc)
    {
        double unused = 0.0;
        RowDot<VT, IT, 1>::run(s, e, lane, val, col, a, a, acc, unused);
    }
};

template <>
struct RowDot1<float, unsigned short, 2> {
    __device__ __forceinline__ static void run(int s, int e, int lane, const float *__restrict__ val,
                                               const unsigned short *__restrict__ col,
                                               const double *__restrict__ a, double &acc)
    {
        double unused = 0.0;
        row_dot_coalesced<false>(s, e, lane, val, col, a, a, acc, unused);
    }
};

template <typename VT, typename IT, int NS>
struct RowDot {
    __device__ __forceinline__ static void run(int s, int e, int lane, const VT *__restrict__ val,
                                               const IT *__restrict__ col, const double *__restrict__ a,
                                               const double *__restrict__ b, double &acc0, double &acc1)
    {
        for (int q = s + 1 + lane; q < e; q += 32) {
            const double g = (double)val[q];
            const int c = (int)col[q];
            acc0 += g * a[c];
            if (NS == 2) acc1 += g * b[c];
        }
    }
};

// one row of the SpMV below
template <typename VT, typename IT, int NS>
__device__ __forceinline__ void spmv_row(const FusedArgs &a, int row, int s, int e, int lane,
                                         const VT *__restrict__ val, const IT *__restrict__ col, const double *v0,
                                         const double *vs0, const double *v1, const double *vs1, double *o0,
                                         double *o1, bool act0, bool act1, bool residual)
{
    // the row's values and positions toward L2 at once (one 128-byte line
    // per lane for each, the first 1024 entries): the loop below walks the
    // row in 256-entry steps whose loads then wait on L2 instead of DRAM
    {
        const char *pv = reinterpret_cast<const char *>(val + s) + 128 * lane;
        const char *pc = reinterpret_cast<const char *>(col + s) + 128 * lane;
        if (pv < reinterpret_cast<const char *>(val + e)) asm volatile("prefetch.global.L2 [%0];" ::"l"(pv));
        if (pc < reinterpret_cast<const char *>(col + e)) asm volatile("prefetch.global.L2 [%0];" ::"l"(pc));
    }
    double acc0 = 0.0, acc1 = 0.0;
    const double gd = (double)val[s];
    // the row's scalars for the epilogue, loaded before the sum (lane 0)
    double f0 = 0.0, f1 = 0.0, r0 = 0.0, r1 = 0.0;
    if (lane == 0) {
        acc0 = act0 ? gd * v0[row] : 0.0;
        if (NS == 2) acc1 = act1 ? gd * v1[row] : 0.0;
        if (act0) {
            const FusedSys &S = a.sys[0];
            f0 = (1.0 + S.dvec[row]) * 0.5 * (S.hrow ? S.hrow[row] : S.h);
            r0 = residual ? S.rhs[row] : 0.0;
        }
        if (NS == 2 && act1) {
            const FusedSys &S = a.sys[1];
            f1 = (1.0 + S.dvec[row]) * 0.5 * (S.hrow ? S.hrow[row] : S.h);
            r1 = residual ? S.rhs[row] : 0.0;
        }
    }
    if (NS == 2 && act0 && act1)
        RowDot<VT, IT, 2>::run(s, e, lane, val, col, vs0, vs1, acc0, acc1);
    else if (act0)
        RowDot1<VT, IT, NS>::run(s, e, lane, val, col, vs0, acc0);
    else if (NS == 2 && act1)
        RowDot1<VT, IT, NS>::run(s, e, lane, val, col, vs1, acc1);
    acc0 = warp_sum(acc0);
    if (NS == 2) acc1 = warp_sum(acc1);
    if (lane == 0) {
        // acc includes G_ii v_i; y = v_i + (1 + d_i)/2 h (G v)_i
        if (act0) {
            const double y = v0[row] + f0 * acc0;
            o0[row] = residual ? r0 - y : y;
        }
        if (NS == 2 && act1) {
            const double y = v1[row] + f1 * acc1;
            o1[row] = residual ? r1 - y : y;
        }
    }
}

// out_s[row] = v_s[row] + (1 + d_s)/2 h_s (G v_s)[row] (sign -1: rhs_s - that),
// one warp per row.  The CTA takes the rows in cell-sorted order, one per
// warp per grab, from the pass's counter: its warps work on consecutive
// sorted positions (spatial neighbours, whose gathers from the cell-sorted
// vector share a few kilobytes), and SMs that run slower (the per-CTA times
// of a static split differ by up to 40 %) simply take fewer rows; the tail is
// one row per warp.  The next grab is issued before the current rows are
// summed (double-buffered in shared memory, one CTA barrier per grab).  Each
// row is summed by one warp in a fixed order, so w does not depend on which
// CTA took it; the dots over w that follow use the static row partition, so
// results stay bit-identical run to run.
template <typename VT, typename IT, int NS>
__device__ __forceinline__ void spmv_rows(const FusedArgs &a, int *ctr, const double *v0, const double *vs0,
                                          const double *v1, const double *vs1, double *o0, double *o1, bool act0,
                                          bool act1, bool residual)
{
    __shared__ int grab[2];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const VT *val = static_cast<const VT *>(a.vals);
    const IT *col = static_cast<const IT *>(a.cols);
    if (threadIdx.x == 0) grab[0] = atomicAdd(ctr, nw);
    __syncthreads();
    int buf = 0;
    int g = grab[0];
    while (g < a.n) {
        if (threadIdx.x == 0) grab[buf ^ 1] = atomicAdd(ctr, nw);
        const int k = g + wid;
        if (k < a.n) {
            const int2 se = a.srow[k]; // loaded beside sorted[k], not after it
            spmv_row<VT, IT, NS>(a, a.sorted[k], se.x, se.y, lane, val, col, v0, vs0, v1, vs1, o0, o1, act0, act1,
                                 residual);
        }
        __syncthreads();
        buf ^= 1;
        g = grab[buf];
    }
}

// Per-CTA partial dots over the CTA's rows r0 .. r1-1: task t = (s, k) for
// s < NS active and k < cnt[s]; vector k is V_s[k] (or w_s itself for
// k == kw[s]: |w|^2).  One warp per task, lanes strided over the rows.
template <int NS>
__device__ __forceinline__ void partial_dots(const FusedArgs &a, int r0, int r1, int n, const int *cnt,
                                             const int *kw, double *part_pass)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ntask = cnt[0] + (NS == 2 ? cnt[1] : 0);
    for (int t = wid; t < ntask; t += nw) {
        const int s = (NS == 2 && t >= cnt[0]) ? 1 : 0;
        const int k = s ? t - cnt[0] : t;
        const FusedSys &S = a.sys[s];
        const double *u = k == kw[s] ? S.w : S.V + (size_t)k * n;
        double acc = 0.0;
        for (int i = r0 + lane; i < r1; i += 32) acc += u[i] * S.w[i];
        acc = warp_sum(acc);
        if (lane == 0) part_pass[((size_t)s * kKM + k) * gridDim.x + blockIdx.x] = acc;
    }
}

// sums[s][k] = sum over the CTAs of the partials (fixed order: the same in
// every CTA)
template <int NS>
__device__ __forceinline__ void reduce_partials(const double *part_pass, const int *cnt, double (*sums)[kKM + 1])
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nb = gridDim.x;
    const int ntask = cnt[0] + (NS == 2 ? cnt[1] : 0);
    for (int t = wid; t < ntask; t += nw) {
        const int s = (NS == 2 && t >= cnt[0]) ? 1 : 0;
        const int k = s ? t - cnt[0] : t;
        const double *p = part_pass + ((size_t)s * kKM + k) * nb;
        double acc = 0.0;
        for (int b = lane; b < nb; b += 32) acc += p[b];
        acc = warp_sum(acc);
        if (lane == 0) sums[s][k] = acc;
    }
}

template <typename VT, typename IT, int NS>
__global__ void __launch_bounds__(kThreads, 2) fused_gmres_kernel(FusedArgs a)
{
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    const int n = a.n, m = a.m;
    const int nb = gridDim.x, tid = threadIdx.x;
    const int chunk = (n + nb - 1) / nb;
    const int r0 = min(n, (int)blockIdx.x * chunk), r1 = min(n, r0 + chunk);
    double *pass0 = a.part, *pass1 = a.part + (size_t)2 * nb * kKM;

    __shared__ double H[NS][kKM][kKM]; // rotated Hessenberg, H[row][col]
    __shared__ double cs[NS][kKM], sn[NS][kKM], gv[NS][kKM + 1], yv[NS][kKM];
    __shared__ double c1[NS][kKM + 1], c2[NS][kKM + 1];
    __shared__ double beta0[NS], nrm[NS];
    __shared__ int conv[NS], act[NS], kcyc[NS], total[NS], bad[NS];
    __shared__ int cnt[2], kw[2];

    // ---- start: x = 0, beta0 = |rhs|, V_0 = rhs / beta0
    for (int s = 0; s < NS; ++s)
        for (int i = r0 + tid; i < r1; i += blockDim.x) a.sys[s].x[i] = 0.0;
    {
        const int lane = tid & 31, wid = tid >> 5;
        if (wid < NS) {
            const FusedSys &S = a.sys[wid];
            double acc = 0.0;
            for (int i = r0 + lane; i < r1; i += 32) acc += S.rhs[i] * S.rhs[i];
            acc = warp_sum(acc);
            if (lane == 0) pass0[(size_t)wid * kKM * nb + blockIdx.x] = acc;
        }
    }
    if (tid < 2) {
        cnt[tid] = tid < NS ? 1 : 0;
        kw[tid] = -1;
    }
    int spass = 0; // SpMV passes so far (the same in every CTA)
    if (blockIdx.x == 0 && tid == 0) a.ctr[0] = 0;
    grid.sync();
    reduce_partials<NS>(pass0, cnt, c1);
    __syncthreads();
    if (tid < NS) {
        const double b0 = sqrt(c1[tid][0]);
        beta0[tid] = b0;
        nrm[tid] = b0;
        bad[tid] = isfinite(b0) ? 0 : 1;
        conv[tid] = (b0 == 0.0 || bad[tid]) ? 1 : 0;
        total[tid] = 0;
    }
    __syncthreads();
    for (int s = 0; s < NS; ++s) {
        if (conv[s]) continue;
        const FusedSys &S = a.sys[s];
        const double inv = 1.0 / nrm[s];
        for (int i = r0 + tid; i < r1; i += blockDim.x) S.V[i] = S.rhs[i] * inv;
    }
    grid.sync();

    for (;;) { // restart cycles
        if (tid < NS) {
            act[tid] = (!conv[tid] && !bad[tid] && total[tid] < a.max_it) ? 1 : 0;
            kcyc[tid] = 0;
            for (int q = 0; q <= m; ++q) gv[tid][q] = 0.0;
            gv[tid][0] = nrm[tid];
        }
        __syncthreads();
        for (int j = 0; j < m; ++j) {
            bool any = false;
            for (int s = 0; s < NS; ++s) any |= act[s] != 0;
            if (!any) break;
            // P1: z = M^-1 V_j, in the user and the cell-sorted order
            for (int s = 0; s < NS; ++s) {
                if (!act[s]) continue;
                const FusedSys &S = a.sys[s];
                const double *vj = S.V + (size_t)j * n;
                for (int k = r0 + tid; k < r1; k += blockDim.x) {
                    const int i = a.sorted[k];
                    const double zi = block_row(S, i, vj);
                    S.zs[k] = zi;
                    S.z[i] = zi;
                }
            }
            grid.sync();
            // P2: w = J z (rows taken from the pass's counter), then the
            // partial dots V_k . w (k <= j) over the CTA's own rows
            if (blockIdx.x == 0 && tid == 0) a.ctr[(spass + 1) & (kPasses - 1)] = 0;
            spmv_rows<VT, IT, NS>(a, a.ctr + (spass & (kPasses - 1)), a.sys[0].z, a.sys[0].zs,
                                  NS == 2 ? a.sys[1].z : nullptr, NS == 2 ? a.sys[1].zs : nullptr, a.sys[0].w,
                                  NS == 2 ? a.sys[1].w : nullptr, act[0] != 0, NS == 2 && act[NS - 1] != 0, false);
            ++spass;
            if (tid < 2) {
                cnt[tid] = (tid < NS && act[tid]) ? j + 1 : 0;
                kw[tid] = -1;
            }
            grid.sync();
            partial_dots<NS>(a, r0, r1, n, cnt, kw, pass0);
            grid.sync();
            // P3: c1; w -= V c1; partial dots V_k . w and |w|^2
            reduce_partials<NS>(pass0, cnt, c1);
            __syncthreads();
            for (int s = 0; s < NS; ++s) {
                if (!act[s]) continue;
                const FusedSys &S = a.sys[s];
                for (int i = r0 + tid; i < r1; i += blockDim.x) {
                    double u = 0.0;
                    for (int k = 0; k <= j; ++k) u += S.V[(size_t)k * n + i] * c1[s][k];
                    S.w[i] -= u;
                }
            }
            if (tid < 2) {
                cnt[tid] = (tid < NS && act[tid]) ? j + 2 : 0;
                kw[tid] = j + 1;
            }
            __syncthreads();
            partial_dots<NS>(a, r0, r1, n, cnt, kw, pass1);
            grid.sync();
            // P4: c2, |w1|^2; w -= V c2; V_{j+1} = w / |w|; rotation and test
            reduce_partials<NS>(pass1, cnt, c2);
            __syncthreads();
            if (tid < NS && act[tid]) {
                double cc = 0.0;
                for (int k = 0; k <= j; ++k) cc += c2[tid][k] * c2[tid][k];
                nrm[tid] = fmax(c2[tid][j + 1] - cc, 0.0);
            }
            __syncthreads();
            for (int s = 0; s < NS; ++s) {
                if (!act[s]) continue;
                const FusedSys &S = a.sys[s];
                const double nr = nrm[s];
                const double inv = nr > 0.0 ? rsqrt(nr) : 0.0;
                double *vn = S.V + (size_t)(j + 1) * n;
                for (int i = r0 + tid; i < r1; i += blockDim.x) {
                    double u = 0.0;
                    for (int k = 0; k <= j; ++k) u += S.V[(size_t)k * n + i] * c2[s][k];
                    const double wn = S.w[i] - u;
                    vn[i] = wn * inv;
                }
            }
            if (tid < NS && act[tid]) {
                const int s = tid;
                const double hn = sqrt(nrm[s]);
                for (int i = 0; i <= j; ++i) H[s][i][j] = c1[s][i] + c2[s][i];
                for (int i = 0; i < j; ++i) {
                    const double x = H[s][i][j], y = H[s][i + 1][j];
                    H[s][i][j] = cs[s][i] * x + sn[s][i] * y;
                    H[s][i + 1][j] = -sn[s][i] * x + cs[s][i] * y;
                }
                const double x = H[s][j][j];
                const double rr = hypot(x, hn);
                cs[s][j] = rr > 0.0 ? x / rr : 1.0;
                sn[s][j] = rr > 0.0 ? hn / rr : 0.0;
                H[s][j][j] = rr;
                gv[s][j + 1] = -sn[s][j] * gv[s][j];
                gv[s][j] = cs[s][j] * gv[s][j];
                total[s] += 1;
                kcyc[s] = j + 1;
                if (!isfinite(hn) || !isfinite(gv[s][j + 1])) {
                    bad[s] = 1;
                    act[s] = 0;
                } else if (fabs(gv[s][j + 1]) <= a.tol * beta0[s] || hn == 0.0) {
                    conv[s] = 1;
                    act[s] = 0;
                } else if (total[s] >= a.max_it) {
                    act[s] = 0;
                }
            }
            __syncthreads();
            bool more = false;
            for (int s = 0; s < NS; ++s) more |= act[s] != 0;
            if (more && j + 1 < m) grid.sync(); // V_{j+1} complete before P1 reads its block members
        }
        // end of cycle: y = R^-1 g, u = V y (into w), x += M^-1 u
        if (tid < NS) {
            const int s = tid, k = kcyc[s];
            for (int i = k - 1; i >= 0; --i) {
                double t = gv[s][i];
                for (int q = i + 1; q < k; ++q) t -= H[s][i][q] * yv[s][q];
                yv[s][i] = t / H[s][i][i];
            }
        }
        __syncthreads();
        for (int s = 0; s < NS; ++s) {
            if (kcyc[s] == 0 || bad[s]) continue;
            const FusedSys &S = a.sys[s];
            for (int i = r0 + tid; i < r1; i += blockDim.x) {
                double u = 0.0;
                for (int k = 0; k < kcyc[s]; ++k) u += S.V[(size_t)k * n + i] * yv[s][k];
                S.w[i] = u;
            }
        }
        grid.sync();
        for (int s = 0; s < NS; ++s) {
            if (kcyc[s] == 0 || bad[s]) continue;
            const FusedSys &S = a.sys[s];
            for (int i = r0 + tid; i < r1; i += blockDim.x) S.x[i] += block_row(S, i, S.w);
        }
        bool again = false;
        for (int s = 0; s < NS; ++s) again |= !conv[s] && !bad[s] && total[s] < a.max_it;
        if (!again) break;
        // restart from the true residual r = rhs - J x of the unconverged systems
        grid.sync();
        __shared__ int rs[2];
        if (tid < 2) rs[tid] = tid < NS ? (!conv[tid] && !bad[tid] && total[tid] < a.max_it) : 0;
        __syncthreads();
        for (int s = 0; s < NS; ++s) {
            if (!rs[s]) continue;
            const FusedSys &S = a.sys[s];
            for (int k = r0 + tid; k < r1; k += blockDim.x) S.zs[k] = S.x[a.sorted[k]];
        }
        grid.sync();
        if (blockIdx.x == 0 && tid == 0) a.ctr[(spass + 1) & (kPasses - 1)] = 0;
        spmv_rows<VT, IT, NS>(a, a.ctr + (spass & (kPasses - 1)), a.sys[0].x, a.sys[0].zs,
                              NS == 2 ? a.sys[1].x : nullptr, NS == 2 ? a.sys[1].zs : nullptr, a.sys[0].w,
                              NS == 2 ? a.sys[1].w : nullptr, rs[0] != 0, NS == 2 && rs[NS - 1] != 0, true);
        ++spass;
        if (tid < 2) {
            cnt[tid] = (tid < NS && rs[tid]) ? 1 : 0;
            kw[tid] = 0;
        }
        grid.sync();
        partial_dots<NS>(a, r0, r1, n, cnt, kw, pass0);
        grid.sync();
        reduce_partials<NS>(pass0, cnt, c1);
        __syncthreads();
        if (tid < NS && rs[tid]) {
            const double b = sqrt(c1[tid][0]);
            nrm[tid] = b;
            if (!isfinite(b)) bad[tid] = 1;
            else if (b <= a.tol * beta0[tid]) conv[tid] = 1;
        }
        __syncthreads();
        for (int s = 0; s < NS; ++s) {
            if (!rs[s] || conv[s] || bad[s]) continue;
            const FusedSys &S = a.sys[s];
            const double inv = 1.0 / nrm[s];
            for (int i = r0 + tid; i < r1; i += blockDim.x) S.V[i] = S.w[i] * inv;
        }
        grid.sync();
    }
    if (blockIdx.x == 0 && tid < NS) {
        const int s = tid;
        double *st = a.sys[s].status;
        st[0] = (double)total[s];
        st[1] = conv[s] && !bad[s] ? 1.0 : 0.0;
        st[2] = beta0[s] > 0.0 ? fabs(gv[s][kcyc[s]]) / beta0[s] : 0.0;
        st[3] = bad[s] ? 1.0 : 0.0;
    }
}

// (start, end) of the row at each cell-sorted position
__global__ void sorted_rows_kernel(int n, const int *__restrict__ sorted, const int *__restrict__ rowptr,
                                   int2 *__restrict__ srow)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int r = sorted[k];
    srow[k] = make_int2(rowptr[r], rowptr[r + 1]);
}

template <typename VT, typename IT, int NS>
const void *kernel_ptr()
{
    return (const void *)fused_gmres_kernel<VT, IT, NS>;
}

const void *pick_kernel(bool valf, bool col16, int ns)
{
    if (valf) {
        if (col16) return ns == 2 ? kernel_ptr<float, unsigned short, 2>() : kernel_ptr<float, unsigned short, 1>();
        return ns == 2 ? kernel_ptr<float, int, 2>() : kernel_ptr<float, int, 1>();
    }
    if (col16) return ns == 2 ? kernel_ptr<double, unsigned short, 2>() : kernel_ptr<double, unsigned short, 1>();
    return ns == 2 ? kernel_ptr<double, int, 2>() : kernel_ptr<double, int, 1>();
}

} // namespace

// Co-resident CTAs of the fused kernel on this device (0: not launchable
// cooperatively); cached per kernel form.
static int fused_grid(const Engine &e, const void *kern)
{
    int coop = 0, sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, e.device) != cudaSuccess || !coop) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e.device) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0) != cudaSuccess) return 0;
    per_sm = per_sm > 2 ? 2 : per_sm;
    return per_sm * sms;
}

bool fused_supported(const Engine &e)
{
    return e.col_s_valid && e.restart <= kKM - 1 &&
           fused_grid(e, pick_kernel(e.valf, e.col_s16_valid, 1)) > 0;
}

int fused_alloc(Engine &e, int ns)
{
    const size_t n = (size_t)e.n;
    if (!e.d_fpart) {
        if (cudaMalloc(&e.d_fpart, sizeof(double) * 2 * 2 * 1024 * kKM) != cudaSuccess) return SDDDST_ERR_NOMEM;
        if (cudaMalloc(&e.d_fstatus, sizeof(double) * 4 * kStatusSlots) != cudaSuccess) return SDDDST_ERR_NOMEM;
        if (cudaMalloc(&e.d_fctr, sizeof(int) * kPasses) != cudaSuccess) return SDDDST_ERR_NOMEM;
        if (cudaMalloc(&e.d_fsrow, sizeof(int2) * (size_t)e.n) != cudaSuccess) return SDDDST_ERR_NOMEM;
        if (cudaMallocHost(&e.h_fstatus, sizeof(double) * 4 * kStatusSlots) != cudaSuccess) return SDDDST_ERR_NOMEM;
    }
    if (ns == 2 && !e.d_V2) {
        if (cudaMalloc(&e.d_V2, sizeof(double) * (e.restart + 1) * n) != cudaSuccess) return SDDDST_ERR_NOMEM;
        double **v[] = {&e.d_w2, &e.d_z2, &e.d_zs2, &e.d_gI, &e.d_solI, &e.d_dvecI, &e.d_vsI};
        for (double **p : v)
            if (cudaMalloc(p, sizeof(double) * n) != cudaSuccess) return SDDDST_ERR_NOMEM;
        if (precond_alloc(e, e.pc2)) return SDDDST_ERR_NOMEM;
    }
    return 0;
}

void fused_free(Engine &e)
{
    double *bufs[] = {e.d_fpart, e.d_fstatus, e.d_V2, e.d_w2, e.d_z2, e.d_zs2, e.d_gI, e.d_solI, e.d_dvecI, e.d_vsI};
    for (double *b : bufs)
        if (b) cudaFree(b);
    if (e.d_fctr) cudaFree(e.d_fctr);
    if (e.d_fsrow) cudaFree(e.d_fsrow);
    if (e.h_fstatus) cudaFreeHost(e.h_fstatus);
}

// Solves J(h_s) x_s = rhs_s for ns (1 or 2) systems sharing the assembled G,
// each preconditioned by its cluster inverse pcs[s], in one cooperative launch;
// conv[s] receives 1 where system s reached the residual target.  Returns
// SDDDST_ERR_NONFINITE when a Krylov quantity is not finite.
int fused_gmres(Engine &e, int ns, const double *h, const double *const *dvec, const double *const *rhs,
                double *const *x, const Cluster *const *pcs, int *conv, bool defer, int slot)
{
    if (int rc = fused_alloc(e, ns)) {
        e.err = "fused solve: allocation failed";
        return rc;
    }
    FusedArgs a{};
    a.n = e.n;
    a.m = e.restart;
    a.max_it = e.prm.max_iters > 0 ? e.prm.max_iters : 1000;
    a.tol = e.prm.solver_tol > 0 ? e.prm.solver_tol : 1e-13;
    a.rowptr = e.d_rowptr;
    a.cols = e.col_s16_valid ? (const void *)e.d_col_s16 : (const void *)e.d_col_s;
    a.vals = e.valf ? (const void *)e.d_valf : (const void *)e.d_val;
    a.sorted = e.spmv_sorted;
    a.part = e.d_fpart;
    a.ctr = e.d_fctr;
    sorted_rows_kernel<<<(e.n + 255) / 256, 256, 0, e.st>>>(e.n, e.spmv_sorted, e.d_rowptr, e.d_fsrow);
    e.launches++;
    a.srow = e.d_fsrow;
    double *Vs[2] = {e.d_V, e.d_V2};
    double *ws[2] = {e.d_w, e.d_w2};
    double *zs[2] = {e.d_z, e.d_z2};
    double *zss[2] = {e.d_vsort, e.d_zs2};
    for (int s = 0; s < ns; ++s) {
        FusedSys &S = a.sys[s];
        const Cluster &c = *pcs[s];
        S.h = h[s];
        S.hrow = e.d_hrow;
        S.dvec = dvec[s];
        S.rhs = rhs[s];
        S.x = x[s];
        S.V = Vs[s];
        S.w = ws[s];
        S.z = zs[s];
        S.zs = zss[s];
        S.blk_of = c.blk_of;
        S.loc = c.loc;
        S.bstart = c.bstart;
        S.blen = c.blen;
        S.members = c.members;
        S.off = c.off;
        S.binv = c.binv;
        S.status = e.d_fstatus + 4 * (slot + s);
    }
    if (ns == 1) a.sys[1] = a.sys[0];
    const void *kern = pick_kernel(e.valf, e.col_s16_valid, ns);
    const int grid = fused_grid(e, kern);
    if (grid <= 0 || grid > 1024) {
        e.err = "fused solve: cooperative launch not available";
        return SDDDST_ERR_CUDA;
    }
    void *args[] = {&a};
    cudaError_t ce = cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kThreads), args, 0, e.st);
    if (ce != cudaSuccess) {
        e.err = std::string("fused solve launch: ") + cudaGetErrorString(ce);
        return SDDDST_ERR_CUDA;
    }
    e.launches++;
    if (defer) return 0;
    cudaMemcpyAsync(e.h_fstatus, e.d_fstatus + 4 * slot, sizeof(double) * 4 * ns, cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("fused solve")) return rc;
    int res = 0;
    for (int s = 0; s < ns; ++s) {
        const double *st = e.h_fstatus + 4 * s;
        const int it = (int)st[0];
        e.solves++;
        e.iterations += it;
        e.last_iters = it;
        e.last_resid = st[2];
        conv[s] = st[1] != 0.0 ? 1 : 0;
        if (st[3] != 0.0) {
            e.err = "solve: non-finite Krylov vector";
            res = SDDDST_ERR_NONFINITE;
        }
    }
    return res;
}

} // namespace sd
