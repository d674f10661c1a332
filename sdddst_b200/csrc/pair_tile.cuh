// Tile bodies of the O(N^2) velocity pair sum, shared by the single-system
// kernels (speeds.cu) and the batched kernels (batch.cu).  Reference:
// Simulation::calculateSpeeds, src/simulation.cpp:86-131.
#pragma once

#include "common.cuh"
#include "field_f32.cuh"
#include "field_f64.cuh"
#include "tabulated_field.cuh"

namespace sd {

// Field of the FP64 tile: the analytic periodic sum, or the tabulated field
// (closed-form image-free term plus the interpolated smooth remainder).
struct AnalyticField64 {
    __device__ __forceinline__ double xy(double dx, double dy) const { return tau_xy_f64(dx, dy); }
};
struct TabulatedField64 {
    const double *rem; // remainder table of tau_xy
    __device__ __forceinline__ double xy(double dx, double dy) const
    {
        return tau0_xy(dx, dy) + tab_interp(rem, dx, dy);
    }
};

// One T x T tile (I, J), I <= J, of the FP64 pair sum over a system of n
// dislocations at x, y, b (see the file comment for the partial-sum layout).
template <int T, class Field = AnalyticField64>
__device__ __forceinline__ void pair_tile_f64(const double *__restrict__ x, const double *__restrict__ y,
                                              const double *__restrict__ b, int n, int I, int J,
                                              double *__restrict__ part, unsigned long long *__restrict__ minr2,
                                              double r2_track, const Field fld = Field())
{
    constexpr int W = T / 32;
    __shared__ double sx[T], sy[T], sb[T];
    __shared__ double tbuf[W][32][33];
    __shared__ double colsum[W][T];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j0 = J * T;
    {
        int j = j0 + tid;
        bool ok = j < n;
        sx[tid] = ok ? x[j] : 0.0;
        sy[tid] = ok ? y[j] : 0.0;
        sb[tid] = ok ? b[j] : 0.0;
    }
    const int i = I * T + tid;
    const bool row_ok = i < n;
    const double xi = row_ok ? x[i] : 0.0;
    const double yi = row_ok ? y[i] : 0.0;
    const double bi = row_ok ? b[i] : 0.0;
    const bool diag = (I == J);
    __syncthreads();

    double acc = 0.0;
    for (int c0 = 0; c0 < T; c0 += 32) {
#pragma unroll 2
        for (int k = 0; k < 32; ++k) {
            const int jj = c0 + k;
            const bool valid = row_ok && (j0 + jj < n) && (!diag || jj > tid);
            double dx = wrap_half(xi - sx[jj]);
            double dy = wrap_half(yi - sy[jj]);
            double r2 = r2_exact(dx, dy);
            if (!valid) {
                dx = 0.25;
                dy = 0.25;
            }
            double t = bi * sb[jj] * fld.xy(dx, dy);
            t = valid ? t : 0.0;
            acc += t;
            if (valid && r2 < r2_track) { // rare: only pairs that can set a tolerance
                atomic_min_nonneg(&minr2[i], r2);
                atomic_min_nonneg(&minr2[j0 + jj], r2);
            }
            tbuf[warp][k][lane] = t;
        }
        __syncwarp();
        double cs = 0.0;
#pragma unroll 8
        for (int m = 0; m < 32; ++m) cs += tbuf[warp][lane][m];
        colsum[warp][c0 + lane] = cs;
        __syncwarp();
    }
    __syncthreads();
    double ctot = 0.0;
#pragma unroll
    for (int w = 0; w < W; ++w) ctot += colsum[w][tid];

    if (diag) {
        if (row_ok) part[(size_t)I * n + i] = acc - ctot;
    } else {
        if (row_ok) part[(size_t)J * n + i] = acc;
        if (j0 + tid < n) part[(size_t)I * n + j0 + tid] = -ctot;
    }
}


// Minimum-image separation of two FP64 coordinates: d - rint(d), with rint
// as the add/subtract of 1.5 * 2^52 (exact round-to-nearest-even for
// |d| < 2^51), two FP64 adds instead of a rounding instruction.
__device__ __forceinline__ double min_image(double d)
{
    const double m = 6755399441055744.0;
    return d - __dadd_rn(__dadd_rn(d, m), -m);
}

// Mixed-precision tiles.  Separations in FP64, rounded once to FP32: dx as
// the minimum-image difference, sin(pi dy) as s_i c_j - c_i s_j from
// per-dislocation s = sin(pi y), c = cos(pi y) (FP64, formed once per tile
// and dislocation).  Field terms in packed FP32 for two columns at a time
// (tau_xy_f32x2, which returns tau2 = tau_xy / pi^2); row and column partials
// summed in FP32 over 16 terms, then carried in FP64:
//   row i:    sum_j (pi^2 b_j) tau2_ij,  times b_i at the end;
//   column j: sum_i (pi^2 b_i) tau2_ij,  times b_j at the end.
// Interior tiles (I < J, full blocks) skip every validity test.
template <int T, bool kChecked>
__device__ __forceinline__ void f32_tile_body(const double *sx, const double *sy, const double *ssn,
                                              const double *scs, const float *sbp, const float *brow, double xi,
                                              double yi, double si, double ci, int n, int j0, int tid, bool row_ok,
                                              bool diag, int i, float *tb, double *colsum_w, double &acc,
                                              unsigned long long *minr2, float r2_track, float s_track)
{
    const int lane = tid & 31;
    for (int c0 = 0; c0 < T; c0 += 32) {
        float2 racc = f2c(0.0f);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int jj = c0 + 2 * m;
            const double2 X = *reinterpret_cast<const double2 *>(sx + jj);
            const double2 S = *reinterpret_cast<const double2 *>(ssn + jj);
            const double2 C = *reinterpret_cast<const double2 *>(scs + jj);
            float2 dx = make_float2(__double2float_rn(min_image(xi - X.x)), __double2float_rn(min_image(xi - X.y)));
            float2 sn = make_float2(__double2float_rn(fma(si, C.x, -ci * S.x)),
                                    __double2float_rn(fma(si, C.y, -ci * S.y)));
            bool va = true, vb = true;
            if (kChecked) {
                va = row_ok && (j0 + jj < n) && (!diag || jj > tid);
                vb = row_ok && (j0 + jj + 1 < n) && (!diag || jj + 1 > tid);
                if (!va) {
                    dx.x = 0.25f;
                    sn.x = 0.70710678f;
                }
                if (!vb) {
                    dx.y = 0.25f;
                    sn.y = 0.70710678f;
                }
            }
            float2 s;
            float2 t = tau_xy_f32x2(dx, sn, s);
            if (kChecked) {
                t.x = va ? t.x : 0.0f;
                t.y = vb ? t.y : 0.0f;
            }
            racc = fma2(t, *reinterpret_cast<const float2 *>(sbp + jj), racc);
            if (fminf(s.x, s.y) < s_track) { // rare: pairs that can set a tolerance
                const float dya = __double2float_rn(min_image(yi - sy[jj]));
                const float dyb = __double2float_rn(min_image(yi - sy[jj + 1]));
                const float ra = fmaf(dx.x, dx.x, dya * dya), rb = fmaf(dx.y, dx.y, dyb * dyb);
                if (va && ra < r2_track) {
                    atomic_min_nonneg(&minr2[i], (double)ra);
                    atomic_min_nonneg(&minr2[j0 + jj], (double)ra);
                }
                if (vb && rb < r2_track) {
                    atomic_min_nonneg(&minr2[i], (double)rb);
                    atomic_min_nonneg(&minr2[j0 + jj + 1], (double)rb);
                }
            }
            *reinterpret_cast<float2 *>(tb + m * 66 + 2 * lane) = t;
        }
        acc += (double)racc.x + (double)racc.y;
        __syncwarp();
        // columns c0 + 2 q, c0 + 2 q + 1 (q = lane & 15) over rows 16 h .. 16 h + 15
        // (h = lane >> 4), weighted by pi^2 b of each row; the two row halves meet
        // through a shuffle
        const int q = lane & 15, h = lane >> 4;
        float2 cs = f2c(0.0f);
#pragma unroll
        for (int r = 0; r < 16; ++r)
            cs = fma2(*reinterpret_cast<const float2 *>(tb + q * 66 + 2 * (16 * h + r)),
                      *reinterpret_cast<const float2 *>(brow + 2 * (16 * h + r)), cs);
        const float ox = __shfl_down_sync(0xffffffffu, cs.x, 16);
        const float oy = __shfl_down_sync(0xffffffffu, cs.y, 16);
        if (h == 0)
            *reinterpret_cast<double2 *>(colsum_w + c0 + 2 * q) =
                make_double2((double)cs.x + (double)ox, (double)cs.y + (double)oy);
        __syncwarp();
    }
}

// One T x T tile of the mixed-precision pair sum.
template <int T>
__device__ __forceinline__ void pair_tile_f32(const double *__restrict__ xw, const double *__restrict__ y,
                                              const double *__restrict__ b, int n, int I, int J,
                                              double *__restrict__ part, unsigned long long *__restrict__ minr2,
                                              float r2_track)
{
    constexpr int W = T / 32;
    __shared__ __align__(16) double sx[T];
    __shared__ __align__(16) double sy[T];
    __shared__ __align__(16) double ssn[T];
    __shared__ __align__(16) double scs[T];
    __shared__ __align__(8) float sbp[T];
    __shared__ __align__(8) float brow[W][64];
    __shared__ __align__(8) float tbuf[W][16 * 66];
    __shared__ __align__(16) double colsum[W][T];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int j0 = J * T;
    const double bj = j0 + tid < n ? b[j0 + tid] : 0.0;
    {
        const int j = j0 + tid;
        const bool ok = j < n;
        const double yj = ok ? y[j] : 0.0;
        double sj, cj;
        sincospi(yj, &sj, &cj);
        sx[tid] = ok ? xw[j] : 0.0;
        sy[tid] = yj;
        ssn[tid] = sj;
        scs[tid] = cj;
        sbp[tid] = kPiSqF * (float)bj;
    }
    const int i = I * T + tid;
    const bool row_ok = i < n;
    const double xi = row_ok ? xw[i] : 0.0;
    const double yi = row_ok ? y[i] : 0.0;
    const double bi = row_ok ? b[i] : 0.0;
    double si, ci;
    sincospi(yi, &si, &ci);
    brow[warp][2 * lane] = brow[warp][2 * lane + 1] = kPiSqF * (float)bi;
    const bool diag = (I == J);
    const bool checked = diag || (j0 + T > n) || (I * T + T > n);
    // s = sinh^2(pi dx) + sin^2(pi dy) <= pi^2 r^2 (1 + pi^2 r^2 / 2) for r^2 < 1e-3
    const float s_track = r2_track <= 0.0f ? -1.0f
                          : r2_track < 1e-3f ? kPiSqF * r2_track * (1.0f + kPiSqF * r2_track) * 1.0001f
                                             : 3.0e38f;
    __syncthreads();
    double acc = 0.0;
    if (checked)
        f32_tile_body<T, true>(sx, sy, ssn, scs, sbp, brow[warp], xi, yi, si, ci, n, j0, tid, row_ok, diag, i,
                               tbuf[warp], colsum[warp], acc, minr2, r2_track, s_track);
    else
        f32_tile_body<T, false>(sx, sy, ssn, scs, sbp, brow[warp], xi, yi, si, ci, n, j0, tid, row_ok, diag, i,
                                tbuf[warp], colsum[warp], acc, minr2, r2_track, s_track);
    __syncthreads();
    double ctot = 0.0;
#pragma unroll
    for (int w = 0; w < W; ++w) ctot += colsum[w][tid];
    ctot *= bj;
    acc *= bi;
    if (diag) {
        if (row_ok) part[(size_t)I * n + i] = acc - ctot;
    } else {
        if (row_ok) part[(size_t)J * n + i] = acc;
        if (j0 + tid < n) part[(size_t)I * n + j0 + tid] = -ctot;
    }
}

} // namespace sd
