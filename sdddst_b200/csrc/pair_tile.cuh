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


// Mixed-precision tiles: separations in FP64 from positions pre-wrapped into
// [-0.5, 0.5) (so x_i - x_j lies in (-1, 1) and one rint() gives the minimum
// image), rounded once to FP32; field terms in FP32; row and column sums in
// FP64.  Interior tiles (I < J, full blocks) skip every validity test.
template <int T, bool kChecked>
__device__ __forceinline__ void f32_tile_body(const double *sx, const double *sy, const float *sb, double xi,
                                              double yi, float bi, int n, int j0, int tid, bool row_ok, bool diag,
                                              int i, float (*tb)[33], double *colsum_w, double &acc,
                                              unsigned long long *minr2, float r2_track)
{
    const int lane = tid & 31;
    for (int c0 = 0; c0 < T; c0 += 32) {
#pragma unroll 4
        for (int k = 0; k < 32; ++k) {
            const int jj = c0 + k;
            double dd = xi - sx[jj];
            dd -= rint(dd);
            double ee = yi - sy[jj];
            ee -= rint(ee);
            float dx = __double2float_rn(dd), dy = __double2float_rn(ee);
            bool valid = true;
            if (kChecked) {
                valid = row_ok && (j0 + jj < n) && (!diag || jj > tid);
                if (!valid) {
                    dx = 0.25f;
                    dy = 0.25f;
                }
            }
            float t = bi * sb[jj] * tau_xy_f32(dx, dy);
            if (kChecked) t = valid ? t : 0.0f;
            acc += (double)t;
            const float r2 = fmaf(dx, dx, dy * dy);
            if (r2 < r2_track && valid) { // rare: pairs that can set a tolerance
                atomic_min_nonneg(&minr2[i], (double)r2);
                atomic_min_nonneg(&minr2[j0 + jj], (double)r2);
            }
            tb[k][lane] = t;
        }
        __syncwarp();
        // column partial of this 32-row chunk summed in FP32 (two halves),
        // then carried in FP64
        float c0s = 0.0f, c1s = 0.0f;
#pragma unroll 8
        for (int m = 0; m < 16; ++m) {
            c0s += tb[lane][m];
            c1s += tb[lane][m + 16];
        }
        colsum_w[c0 + lane] = (double)c0s + (double)c1s;
        __syncwarp();
    }
}

// One T x T tile of the mixed-precision pair sum (positions pre-wrapped).
template <int T>
__device__ __forceinline__ void pair_tile_f32(const double *__restrict__ xw, const double *__restrict__ y,
                                              const double *__restrict__ b, int n, int I, int J,
                                              double *__restrict__ part, unsigned long long *__restrict__ minr2,
                                              float r2_track)
{
    constexpr int W = T / 32;
    __shared__ double sx[T], sy[T];
    __shared__ float sb[T];
    __shared__ float tbuf[W][32][33];
    __shared__ double colsum[W][T];

    const int tid = threadIdx.x, warp = tid >> 5;
    const int j0 = J * T;
    {
        const int j = j0 + tid;
        const bool ok = j < n;
        sx[tid] = ok ? xw[j] : 0.0;
        sy[tid] = ok ? y[j] : 0.0;
        sb[tid] = ok ? (float)b[j] : 0.0f;
    }
    const int i = I * T + tid;
    const bool row_ok = i < n;
    const double xi = row_ok ? xw[i] : 0.0;
    const double yi = row_ok ? y[i] : 0.0;
    const float bi = row_ok ? (float)b[i] : 0.0f;
    const bool diag = (I == J);
    const bool checked = diag || (j0 + T > n) || (I * T + T > n);
    __syncthreads();
    double acc = 0.0;
    if (checked)
        f32_tile_body<T, true>(sx, sy, sb, xi, yi, bi, n, j0, tid, row_ok, diag, i, tbuf[warp], colsum[warp], acc,
                               minr2, r2_track);
    else
        f32_tile_body<T, false>(sx, sy, sb, xi, yi, bi, n, j0, tid, row_ok, diag, i, tbuf[warp], colsum[warp], acc,
                                minr2, r2_track);
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


} // namespace sd
