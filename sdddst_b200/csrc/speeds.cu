// O(N^2) velocity pair sum (reference: Simulation::calculateSpeeds,
// src/simulation.cpp:86-131).
//
// Work is split into T x T tiles (I, J), I <= J, over the unique pairs
// i < j (the reference's antisymmetry res[i] += t, res[j] -= t).  A CTA stages
// the J block's x, y, b in shared memory; each thread owns one row i of the
// I block and walks the block's columns.  Row sums stay in registers; column
// sums are transposed through shared memory per 32-column chunk and reduced
// across warps.  Every partial lands in a private slot of part[nblk][N]:
//   part[J][i] <- row partial of tile (I, J) for i in block I
//   part[I][j] <- column partial of tile (I, J) for j in block J
//   part[I][i] <- both partials of the diagonal tile (I, I)
// so no two tiles write the same slot and the final per-dislocation sum over
// the nblk slots runs in a fixed order (bit-reproducible run to run).
//
// The precision handler needs min r^2 per dislocation only below
// 400 prec^2 (updateTolerance, precision_handler.cpp:72-87, acts only when
// r^2/400 < prec^2), so close pairs alone do an atomicMin on the bit pattern.
#include "engine.h"
#include "pair_tile.cuh"

namespace sd {

__device__ __forceinline__ void tile_coords(long t, int &I, int &J)
{
    int j = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long)j * (j + 1) / 2 > t) --j;
    while ((long)(j + 1) * (j + 2) / 2 <= t) ++j;
    J = j;
    I = (int)(t - (long)j * (j + 1) / 2);
}

template <int T, int kMode>
__global__ void __launch_bounds__(T) pair_tiles_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                                       const double *__restrict__ b, int n, int nblk,
                                                       double *__restrict__ part,
                                                       unsigned long long *__restrict__ minr2, double r2_track)
{
    int I, J;
    tile_coords((long)blockIdx.x, I, J);
    pair_tile_f64<T>(x, y, b, n, I, J, part, minr2, r2_track);
}

template <int T>
__global__ void __launch_bounds__(T) pair_tiles_tab_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                                           const double *__restrict__ b, int n, int nblk,
                                                           double *__restrict__ part,
                                                           unsigned long long *__restrict__ minr2, double r2_track,
                                                           const double *__restrict__ rem)
{
    int I, J;
    tile_coords((long)blockIdx.x, I, J);
    pair_tile_f64<T, TabulatedField64>(x, y, b, n, I, J, part, minr2, r2_track, TabulatedField64{rem});
}

template <int T>
__global__ void __launch_bounds__(T) pair_tiles_f32_kernel(const double *__restrict__ xw, const double *__restrict__ y,
                                                           const double *__restrict__ b, int n, int nblk,
                                                           double *__restrict__ part,
                                                           unsigned long long *__restrict__ minr2, float r2_track)
{
    int I, J;
    tile_coords((long)blockIdx.x, I, J);
    pair_tile_f32<T>(xw, y, b, n, I, J, part, minr2, r2_track);
}

__global__ void wrap_kernel(int n, const double *__restrict__ x, double *__restrict__ xw)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xw[i] = wrap_half(x[i]);
}

// Per-dislocation finish: sum of the nblk partials in fixed order, point
// defects (simulation.cpp:111-128), S = pair + defect sum, v = S + b tau_ext
// (simulation.cpp:129), and the tolerance update from min r^2.  A block of
// kFinishGroups warps serves 32 dislocations: warp g sums the g-th quarter of
// the partials (lanes on consecutive dislocations: each load is one 256-byte
// row segment, sixteen in flight per warp), and the quarters are combined in
// order by warp 0.
constexpr int kFinishGroups = 4;

__device__ __forceinline__ void neumaier_add(double &acc, double &comp, double v)
{
    const double t = acc + v;
    comp += fabs(acc) >= fabs(v) ? (acc - t) + v : (v - t) + acc;
    acc = t;
}

__global__ void __launch_bounds__(32 * kFinishGroups)
    speeds_finish_kernel(int n, int nblk, const double *__restrict__ part, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ b, int p,
                         const double *__restrict__ pdx, const double *__restrict__ pdy, double A, double K,
                         double tau_ext, double *__restrict__ S, double *__restrict__ v,
                         const unsigned long long *__restrict__ minr2, double *__restrict__ tol, double prec_sqr,
                         int update_tol, double *__restrict__ minr2_out)
{
    __shared__ double sacc[kFinishGroups][32], scomp[kFinishGroups][32];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    // compensated (Neumaier) FP64 sums of the per-tile partials: the tile
    // partials themselves are FP64 sums of at most one tile's pairs, so the
    // long reduction is this one
    const int per = (nblk + kFinishGroups - 1) / kFinishGroups;
    const int L0 = g * per, L1 = min(nblk, L0 + per);
    double acc = 0.0, comp = 0.0;
    if (i < n) {
#pragma unroll 16
        for (int L = L0; L < L1; ++L) neumaier_add(acc, comp, part[(size_t)L * n + i]);
    }
    sacc[g][lane] = acc;
    scomp[g][lane] = comp;
    __syncthreads();
    if (g != 0 || i >= n) return;
    acc = 0.0;
    comp = 0.0;
#pragma unroll
    for (int k = 0; k < kFinishGroups; ++k) {
        neumaier_add(acc, comp, sacc[k][lane]);
        comp += scomp[k][lane];
    }
    acc += comp;
    double smin = update_tol ? __longlong_as_double((long long)minr2[i]) : 0.0;
    const double xi = x[i], yi = y[i], bi = b[i];
    for (int q = 0; q < p; ++q) {
        double dx = wrap_half(xi - pdx[q]);
        double dy = wrap_half(yi - pdy[q]);
        double s;
        const double f = pd_force_f64(dx, dy, A, K, &s);
        acc -= f * bi;
        if (s < smin) smin = s;
    }
    if (S) S[i] = acc;
    v[i] = acc + bi * tau_ext;
    if (minr2_out) minr2_out[i] = smin;
    if (update_tol) {
        double t = __dmul_rn(__dmul_rn(smin, 0.25), 1e-2); // precision_handler.cpp:74
        double cur = tol[i];
        if (t < prec_sqr && t < cur) tol[i] = (t == 0.0) ? kEps : t;
    }
}

__global__ void add_stress_kernel(int n, const double *__restrict__ S, const double *__restrict__ b, double tau_ext,
                                  double *__restrict__ v)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = S[i] + b[i] * tau_ext;
}

__global__ void fill_u64_kernel(unsigned long long *p, unsigned long long v, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

int pair_tile_size(int n) { return n >= 8192 ? 128 : 64; }

void launch_pair_sum(const Engine &e, const double *x, cudaStream_t st, int mode, double r2_track)
{
    const int n = e.n;
    const int T = pair_tile_size(n);
    const int nblk = (n + T - 1) / T;
    const long tiles = (long)nblk * (nblk + 1) / 2;
    fill_u64_kernel<<<(n + 255) / 256, 256, 0, st>>>(e.d_minr2, 0x7FF0000000000000ull, n);
    if (e.d_tab_xy) { // tabulated field: FP64 tiles whatever the pair-sum mode
        if (T == 128)
            pair_tiles_tab_kernel<128><<<(unsigned)tiles, 128, 0, st>>>(x, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2,
                                                                        r2_track, e.d_tab_xy);
        else
            pair_tiles_tab_kernel<64><<<(unsigned)tiles, 64, 0, st>>>(x, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2,
                                                                      r2_track, e.d_tab_xy);
        return;
    }
    if (mode == 0) {
        if (T == 128)
            pair_tiles_kernel<128, 0><<<(unsigned)tiles, 128, 0, st>>>(x, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2, r2_track);
        else
            pair_tiles_kernel<64, 0><<<(unsigned)tiles, 64, 0, st>>>(x, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2, r2_track);
    } else {
        wrap_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, e.d_xw);
        const float tr = (float)r2_track;
        if (T == 128)
            pair_tiles_f32_kernel<128><<<(unsigned)tiles, 128, 0, st>>>(e.d_xw, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2, tr);
        else
            pair_tiles_f32_kernel<64><<<(unsigned)tiles, 64, 0, st>>>(e.d_xw, e.d_y, e.d_b, n, nblk, e.d_part, e.d_minr2, tr);
    }
}

void launch_speeds_finish(const Engine &e, const double *x, double tau_ext, double *S, double *v, int update_tol,
                          cudaStream_t st)
{
    const int n = e.n;
    const int T = pair_tile_size(n);
    const int nblk = (n + T - 1) / T;
    speeds_finish_kernel<<<(n + 31) / 32, 32 * kFinishGroups, 0, st>>>(n, nblk, e.d_part, x, e.d_y, e.d_b, e.p, e.d_pdx, e.d_pdy,
                                                         e.A, e.KASQR, tau_ext, S, v, e.d_minr2, e.d_tol,
                                                         e.prec * e.prec, update_tol, e.d_minr2_out);
}

void launch_add_stress(const Engine &e, const double *S, double tau_ext, double *v, cudaStream_t st)
{
    add_stress_kernel<<<(e.n + 255) / 256, 256, 0, st>>>(e.n, S, e.d_b, tau_ext, v);
}

// Launches with caller-provided buffers (no engine): FP64 pair sum without
// tolerance tracking, then v = sum + b tau_ext.  `part` must hold
// pair_part_doubles(n) doubles; every slot of it is written before it is read.
void launch_speeds_raw(int n, const double *x, const double *y, const double *b, double tau_ext, double *part,
                       double *v, cudaStream_t st)
{
    const int T = pair_tile_size(n);
    const int nblk = (n + T - 1) / T;
    const long tiles = (long)nblk * (nblk + 1) / 2;
    if (T == 128)
        pair_tiles_kernel<128, 0><<<(unsigned)tiles, 128, 0, st>>>(x, y, b, n, nblk, part, nullptr, 0.0);
    else
        pair_tiles_kernel<64, 0><<<(unsigned)tiles, 64, 0, st>>>(x, y, b, n, nblk, part, nullptr, 0.0);
    speeds_finish_kernel<<<(n + 31) / 32, 32 * kFinishGroups, 0, st>>>(n, nblk, part, x, y, b, 0, nullptr, nullptr, 0.0, 0.0,
                                                         tau_ext, nullptr, v, nullptr, nullptr, 0.0, 0, nullptr);
}

size_t pair_part_doubles(int n)
{
    const int T = pair_tile_size(n);
    const int nblk = (n + T - 1) / T;
    return (size_t)nblk * (size_t)n;
}

} // namespace sd
