// Eigenvalue analysis of a configuration: the reference's --ev-analyzation
// mode (src/main.cpp:36-41 -> TimeSeriesProcessor::run,
// src/time_series_processor.cpp:21-204).
//
//  * The dense Hessian of SpectralDecompositor::decompose
//    (spectral_decompositor.cpp:63-165), FP64, n x n row-major (symmetric, so
//    also column-major): one block per 32 x 32 tile of the lower triangle
//    evaluates b_i b_j xy_diff_x(x_i - x_j, y_i - y_j) once per unordered
//    pair (i > j, the reference's orientation) and stores the tile and its
//    transpose through shared memory, both row-contiguous; then one warp per
//    row sets the diagonal to minus the row's off-diagonal sum minus b_i times
//    the point-defect derivative, whose scaling is the decomposer's own:
//    A = 1.6e-3 / sqrt(defect count), K = 1.65^2 1e6 / 256 n (:76-84).
//  * The eigenpairs by cuSOLVER's divide-and-conquer symmetric eigensolver
//    (the device counterpart of the LAPACKE_dsyevd call at :188): eigenvalues
//    ascending, eigenvector m contiguous at V[m n ..] (column-major output).
//    cuSOLVER and cuBLAS are opened with dlopen on first use, so the rest of
//    the library loads and runs without them.
//  * The observables of :44-89, one block per mode: participation number
//    1 / sum_j v_mj^4, Burgers sum s_m = sum_j v_mj b_j, 1/Gael = s_m^2 / lambda_m.
//  * The eigenvalue derivatives of :93-121 and calculateHessianDerivative
//    (:208-247).  The reference sums V_mi V_mj sum_k v_k dH_ij/dx_k / rate over
//    i, j, k for every mode (n^4 terms).  dH_ij/dx_k vanishes unless two of
//    i, j, k coincide, which collapses sum_k v_k dH_ij/dx_k to
//       M_ij = b_i b_j F(x_i - x_j, y_i - y_j) (v_i - v_j)   (i != j),
//       M_ii = -sum_{j != i} M_ij
//    (F = xy_diff_x2 is odd in the separation, so M is symmetric), and the
//    derivative of mode m to v_m^T M v_m / rate: M by the Hessian's tile and
//    diagonal kernels, W = M V by one cuBLAS DGEMM, a column dot per mode
//    (n^3).  Only a fixed-rate stress protocol has a derivative there; other
//    protocols give zeros, as the reference's type check does.
//  * The correlation matrices of :145-197: the bin (floor((dx + 1/2) S),
//    floor((dy + 1/2) S)) and the sign class of every ordered pair do not
//    depend on the mode and are coded once (one int per pair); then one
//    block per mode accumulates w_i w_j (w = V_m^2) into shared-memory
//    histograms of equal-sign and opposite-sign pairs; the all-pairs
//    histogram is their sum.  A bin index that rounds up to S (dx + 1/2 = 1
//    after rounding; past the reference's arrays) is clamped to S - 1.
#include <dlfcn.h>

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "field_f64.cuh"

namespace sd {

namespace {

constexpr int kTile = 32;

// ---- cuSOLVER / cuBLAS entry points, resolved at run time
struct LinalgApi {
    bool tried = false, ok = false;
    cusolverStatus_t (*dnCreate)(cusolverDnHandle_t *);
    cusolverStatus_t (*dnDestroy)(cusolverDnHandle_t);
    cusolverStatus_t (*dnSetStream)(cusolverDnHandle_t, cudaStream_t);
    cusolverStatus_t (*createParams)(cusolverDnParams_t *);
    cusolverStatus_t (*destroyParams)(cusolverDnParams_t);
    cusolverStatus_t (*syevdBuf)(cusolverDnHandle_t, cusolverDnParams_t, cusolverEigMode_t, cublasFillMode_t,
                                 int64_t, cudaDataType, const void *, int64_t, cudaDataType, const void *,
                                 cudaDataType, size_t *, size_t *);
    cusolverStatus_t (*syevd)(cusolverDnHandle_t, cusolverDnParams_t, cusolverEigMode_t, cublasFillMode_t, int64_t,
                              cudaDataType, void *, int64_t, cudaDataType, void *, cudaDataType, void *, size_t,
                              void *, size_t, int *);
    cublasStatus_t (*blasCreate)(cublasHandle_t *);
    cublasStatus_t (*blasDestroy)(cublasHandle_t);
    cublasStatus_t (*blasSetStream)(cublasHandle_t, cudaStream_t);
    cublasStatus_t (*dgemm)(cublasHandle_t, cublasOperation_t, cublasOperation_t, int, int, int, const double *,
                            const double *, int, const double *, int, const double *, double *, int);
};

LinalgApi g_api;

void *open_lib(const char *name)
{
    // one already in the process (a framework's copy) first, else the system's
    void *h = dlopen(name, RTLD_NOW | RTLD_NOLOAD);
    return h ? h : dlopen(name, RTLD_NOW | RTLD_LOCAL);
}

template <typename F> bool sym(void *h, const char *name, F &f)
{
    f = reinterpret_cast<F>(dlsym(h, name));
    return f != nullptr;
}

bool load_api()
{
    if (g_api.tried) return g_api.ok;
    g_api.tried = true;
    void *s = open_lib("libcusolver.so.11");
    void *b = open_lib("libcublas.so.12");
    if (!s || !b) return false;
    g_api.ok = sym(s, "cusolverDnCreate", g_api.dnCreate) && sym(s, "cusolverDnDestroy", g_api.dnDestroy) &&
               sym(s, "cusolverDnSetStream", g_api.dnSetStream) &&
               sym(s, "cusolverDnCreateParams", g_api.createParams) &&
               sym(s, "cusolverDnDestroyParams", g_api.destroyParams) &&
               sym(s, "cusolverDnXsyevd_bufferSize", g_api.syevdBuf) && sym(s, "cusolverDnXsyevd", g_api.syevd) &&
               sym(b, "cublasCreate_v2", g_api.blasCreate) && sym(b, "cublasDestroy_v2", g_api.blasDestroy) &&
               sym(b, "cublasSetStream_v2", g_api.blasSetStream) && sym(b, "cublasDgemm_v2", g_api.dgemm);
    return g_api.ok;
}

struct EvWork {
    int n = 0;
    double *d_H = nullptr;  // Hessian, then the eigenvectors
    double *d_w = nullptr;  // eigenvalues
    double *d_obs = nullptr; // participation, Burgers sum, 1/Gael, derivative (4 n)
    double *d_M = nullptr, *d_W = nullptr;
    int *d_code = nullptr;
    int code_bins = 0;
    double *d_corr = nullptr;
    size_t corr_cap = 0;
    void *d_work = nullptr;
    size_t work_bytes = 0;
    std::vector<char> h_work;
    int *d_info = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cusolverDnParams_t params = nullptr;
    cublasHandle_t blas = nullptr;
    cudaEvent_t ev[6] = {};
    float ms[5] = {0, 0, 0, 0, 0};
};

// lower-triangle tile k -> (ti, tj), ti >= tj
__device__ __forceinline__ void tri_tile(long k, int &ti, int &tj)
{
    long t = (long)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while (t * (t + 1) / 2 > k) --t;
    while ((t + 1) * (t + 2) / 2 <= k) ++t;
    ti = (int)t;
    tj = (int)(k - t * (t + 1) / 2);
}

// Off-diagonal entries of H (kDeriv false) or M (kDeriv true); the diagonal
// of each diagonal tile is written as 0.  Block 32 x 8.
template <bool kDeriv>
__global__ void __launch_bounds__(256) pair_tiles_kernel(int n, const double *__restrict__ x,
                                                         const double *__restrict__ y, const double *__restrict__ b,
                                                         const double *__restrict__ v, double *__restrict__ H)
{
    __shared__ double tile[kTile][kTile + 1];
    int ti, tj;
    tri_tile(blockIdx.x, ti, tj);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int j = tj * kTile + tx;
    double xj = 0, yj = 0, bj = 0, vj = 0;
    if (j < n) {
        xj = x[j];
        yj = y[j];
        bj = b[j];
        if (kDeriv) vj = v[j];
    }
#pragma unroll
    for (int r = 0; r < kTile / 8; ++r) {
        const int ir = ty + 8 * r, i = ti * kTile + ir;
        double val = 0.0;
        if (i < n && j < n && i > j) {
            const double dx = wrap_half(x[i] - xj), dy = wrap_half(y[i] - yj);
            if (kDeriv)
                val = b[i] * bj * tau_xy_dx2_f64(dx, dy) * (v[i] - vj);
            else
                val = b[i] * bj * tau_xy_dx_f64(dx, dy);
        }
        tile[ir][tx] = val;
    }
    __syncthreads();
    if (ti == tj) {
        // one tile holds both halves: (r, c) = lower value at r > c, its mirror at r < c
#pragma unroll
        for (int r = 0; r < kTile / 8; ++r) {
            const int ir = ty + 8 * r, i = ti * kTile + ir, c = tj * kTile + tx;
            if (i < n && c < n) H[(size_t)i * n + c] = ir > tx ? tile[ir][tx] : ir < tx ? tile[tx][ir] : 0.0;
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < kTile / 8; ++r) {
        const int ir = ty + 8 * r, i = ti * kTile + ir;
        if (i < n && j < n) H[(size_t)i * n + j] = tile[ir][tx];
        // transpose: row tj*32 + ir, column ti*32 + tx
        const int it = tj * kTile + ir, jt = ti * kTile + tx;
        if (it < n && jt < n) H[(size_t)it * n + jt] = tile[tx][ir];
    }
}

// Diagonal: one warp per row, H_ii = -sum_{j != i} H_ij - b_i sum_k pd'(x_i - p_k)
__global__ void diag_kernel(int n, double *__restrict__ H, const double *__restrict__ x,
                            const double *__restrict__ y, const double *__restrict__ b, int p,
                            const double *__restrict__ pdx, const double *__restrict__ pdy, double A, double K)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *row = H + (size_t)warp * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += row[j]; // the diagonal itself is 0 here
    s = warp_sum(s);
    double d = 0.0;
    for (int k = lane; k < p; k += 32)
        d += pd_force_dx_f64(wrap_half(x[warp] - pdx[k]), wrap_half(y[warp] - pdy[k]), A, K);
    d = warp_sum(d);
    if (lane == 0) H[(size_t)warp * n + warp] = -s - b[warp] * d;
}

template <int kThreads> __device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < kThreads / 32 ? sh[threadIdx.x] : 0.0;
        t = warp_sum(t);
    }
    return t; // valid in thread 0
}

// One block per mode: participation number, Burgers sum, 1/Gael.
__global__ void __launch_bounds__(256) observables_kernel(int n, const double *__restrict__ V,
                                                          const double *__restrict__ w, const double *__restrict__ b,
                                                          double *__restrict__ obs)
{
    __shared__ double sh[8];
    const int m = blockIdx.x;
    const double *vm = V + (size_t)m * n;
    double q = 0.0, s = 0.0;
    for (int j = threadIdx.x; j < n; j += 256) {
        const double a = vm[j], a2 = a * a;
        q += a2 * a2;
        s += a * b[j];
    }
    q = block_sum<256>(q, sh);
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) {
        obs[m] = 1.0 / q;
        obs[n + m] = s;
        obs[2 * n + m] = s * s / w[m];
    }
}

// One block per mode: derivative v_m . (M v_m) / rate.
__global__ void __launch_bounds__(256) deriv_dot_kernel(int n, const double *__restrict__ V,
                                                        const double *__restrict__ W, double rate,
                                                        double *__restrict__ out)
{
    __shared__ double sh[8];
    const int m = blockIdx.x;
    const double *vm = V + (size_t)m * n, *wm = W + (size_t)m * n;
    double s = 0.0;
    for (int j = threadIdx.x; j < n; j += 256) s += vm[j] * wm[j];
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) out[m] = s / rate;
}

// Pair codes of the correlation matrices: -1 on the diagonal, else
// 2 (tx S + ty) + (b_i != b_j).
__global__ void pair_code_kernel(int n, int S, const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ b, int *__restrict__ code)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * n) return;
    const int i = (int)(idx / (size_t)n), j = (int)(idx % (size_t)n);
    if (i == j) {
        code[idx] = -1;
        return;
    }
    const double dx = wrap_half(x[i] - x[j]), dy = wrap_half(y[i] - y[j]);
    int tx = (int)floor((dx + 0.5) * S), ty = (int)floor((dy + 0.5) * S);
    tx = min(max(tx, 0), S - 1);
    ty = min(max(ty, 0), S - 1);
    code[idx] = 2 * (tx * S + ty) + (b[i] != b[j] ? 1 : 0);
}

// One block per mode: histograms of w_i w_j over the ordered pairs.
// out[m] = [pp | pn | pp + pn], each S x S.  Shared-memory histograms when
// they fit (kShared), else atomics on the output itself.
template <bool kShared>
__global__ void __launch_bounds__(512) correl_kernel(int n, int S, const double *__restrict__ V,
                                                     const int *__restrict__ code, double *__restrict__ out)
{
    extern __shared__ double hist[];
    const int m = blockIdx.x, SS = S * S;
    const double *vm = V + (size_t)m * n;
    double *o = out + (size_t)m * 3 * SS;
    double *h = kShared ? hist : o;
    if (kShared)
        for (int t = threadIdx.x; t < 2 * SS; t += blockDim.x) hist[t] = 0.0;
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        const double wi = vm[i] * vm[i];
        const int *ci = code + (size_t)i * n;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int c = ci[j];
            if (c < 0) continue;
            const double vj = vm[j];
            atomicAdd(h + (c & 1) * SS + (c >> 1), wi * (vj * vj));
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < SS; t += blockDim.x) {
        const double pp = h[t], pn = h[SS + t];
        if (kShared) {
            o[t] = pp;
            o[SS + t] = pn;
        }
        o[2 * SS + t] = pp + pn;
    }
}

int ensure(double **p, size_t count)
{
    if (*p) return 0;
    return cudaMalloc(p, sizeof(double) * std::max<size_t>(count, 1)) == cudaSuccess ? 0 : SDDDST_ERR_NOMEM;
}

EvWork *work_of(Engine &e)
{
    if (!e.ev) e.ev = new EvWork;
    return static_cast<EvWork *>(e.ev);
}

// tile kernel + diagonal for H (v = nullptr) or M (v = velocities)
void launch_matrix(Engine &e, const double *x, const double *v, double *out, double sdA, double sdK)
{
    const int n = e.n, T = (n + kTile - 1) / kTile;
    const long tiles = (long)T * (T + 1) / 2;
    if (v)
        pair_tiles_kernel<true><<<(unsigned)tiles, dim3(32, 8), 0, e.st>>>(n, x, e.d_y, e.d_b, v, out);
    else
        pair_tiles_kernel<false><<<(unsigned)tiles, dim3(32, 8), 0, e.st>>>(n, x, e.d_y, e.d_b, nullptr, out);
    diag_kernel<<<(n + 7) / 8, 256, 0, e.st>>>(n, out, x, e.d_y, e.d_b, v ? 0 : e.p, e.d_pdx, e.d_pdy, sdA, sdK);
    e.launches += 2;
}

} // namespace

void ev_free(Engine &e)
{
    EvWork *w = static_cast<EvWork *>(e.ev);
    if (!w) return;
    for (double *p : {w->d_H, w->d_w, w->d_obs, w->d_M, w->d_W, w->d_corr})
        if (p) cudaFree(p);
    if (w->d_code) cudaFree(w->d_code);
    if (w->d_work) cudaFree(w->d_work);
    if (w->d_info) cudaFree(w->d_info);
    if (w->params) g_api.destroyParams(w->params);
    if (w->solver) g_api.dnDestroy(w->solver);
    if (w->blas) g_api.blasDestroy(w->blas);
    for (cudaEvent_t ev : w->ev)
        if (ev) cudaEventDestroy(ev);
    delete w;
    e.ev = nullptr;
}

// The Hessian of the configuration x (device; y, b, defects from the engine).
int ev_hessian(Engine &e, const double *x)
{
    EvWork *w = work_of(e);
    const size_t nn = (size_t)e.n * e.n;
    if (ensure(&w->d_H, nn)) {
        e.err = "eigenvalue analysis: Hessian allocation failed";
        return SDDDST_ERR_NOMEM;
    }
    const double sdA = e.p > 0 ? 1e-4 * 16.0 * 1. / std::sqrt((double)e.p) : 0.0;
    const double sdK = e.p > 0 ? 1.65 * 1.65 * 1e6 / 256.0 * (double)e.n : 0.0;
    launch_matrix(e, x, nullptr, w->d_H, sdA, sdK);
    return 0;
}

const double *ev_hessian_ptr(Engine &e) { return e.ev ? static_cast<EvWork *>(e.ev)->d_H : nullptr; }

// Full analysis at x with the velocities v (device, n): eigenpairs in
// d_H / d_w, observables, optional derivatives and correlation matrices.
int ev_analyze(Engine &e, const double *x, const double *v, bool deriv, double rate, int corr_bins)
{
    if (!load_api()) {
        e.err = "eigenvalue analysis: cuSOLVER/cuBLAS (libcusolver.so.11, libcublas.so.12) could not be loaded";
        return SDDDST_ERR_CUDA;
    }
    EvWork *w = work_of(e);
    const int n = e.n;
    const size_t nn = (size_t)n * n;
    if (!w->ev[0])
        for (cudaEvent_t &ev : w->ev) cudaEventCreate(&ev);
    if (!w->solver) {
        if (g_api.dnCreate(&w->solver) != CUSOLVER_STATUS_SUCCESS ||
            g_api.createParams(&w->params) != CUSOLVER_STATUS_SUCCESS ||
            g_api.blasCreate(&w->blas) != CUBLAS_STATUS_SUCCESS) {
            e.err = "eigenvalue analysis: cuSOLVER/cuBLAS handle creation failed";
            return SDDDST_ERR_CUDA;
        }
    }
    g_api.dnSetStream(w->solver, e.st);
    g_api.blasSetStream(w->blas, e.st);
    if (ensure(&w->d_w, n) || ensure(&w->d_obs, 4 * (size_t)n) ||
        (!w->d_info && cudaMalloc(&w->d_info, sizeof(int)) != cudaSuccess)) {
        e.err = "eigenvalue analysis: allocation failed";
        return SDDDST_ERR_NOMEM;
    }
    cudaEventRecord(w->ev[0], e.st);
    if (int rc = ev_hessian(e, x)) return rc;
    cudaEventRecord(w->ev[1], e.st);
    size_t dbytes = 0, hbytes = 0;
    if (g_api.syevdBuf(w->solver, w->params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F, w->d_H,
                       n, CUDA_R_64F, w->d_w, CUDA_R_64F, &dbytes, &hbytes) != CUSOLVER_STATUS_SUCCESS) {
        e.err = "eigenvalue analysis: eigensolver workspace query failed";
        return SDDDST_ERR_CUDA;
    }
    if (dbytes > w->work_bytes) {
        if (w->d_work) cudaFree(w->d_work);
        w->d_work = nullptr;
        w->work_bytes = 0;
        if (cudaMalloc(&w->d_work, dbytes) != cudaSuccess) {
            e.err = "eigenvalue analysis: eigensolver workspace allocation failed";
            return SDDDST_ERR_NOMEM;
        }
        w->work_bytes = dbytes;
    }
    if (w->h_work.size() < hbytes) w->h_work.resize(hbytes);
    if (g_api.syevd(w->solver, w->params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F, w->d_H, n,
                    CUDA_R_64F, w->d_w, CUDA_R_64F, w->d_work, dbytes, hbytes ? w->h_work.data() : nullptr, hbytes,
                    w->d_info) != CUSOLVER_STATUS_SUCCESS) {
        e.err = "eigenvalue analysis: eigensolver launch failed";
        return SDDDST_ERR_CUDA;
    }
    cudaEventRecord(w->ev[2], e.st);
    observables_kernel<<<n, 256, 0, e.st>>>(n, w->d_H, w->d_w, e.d_b, w->d_obs);
    e.launches += 1;
    cudaEventRecord(w->ev[3], e.st);
    if (deriv) {
        if (ensure(&w->d_M, nn) || ensure(&w->d_W, nn)) {
            e.err = "eigenvalue analysis: derivative matrices allocation failed";
            return SDDDST_ERR_NOMEM;
        }
        launch_matrix(e, x, v, w->d_M, 0.0, 0.0);
        const double one = 1.0, zero = 0.0;
        if (g_api.dgemm(w->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, w->d_M, n, w->d_H, n, &zero, w->d_W, n) !=
            CUBLAS_STATUS_SUCCESS) {
            e.err = "eigenvalue analysis: DGEMM failed";
            return SDDDST_ERR_CUDA;
        }
        deriv_dot_kernel<<<n, 256, 0, e.st>>>(n, w->d_H, w->d_W, rate, w->d_obs + 3 * (size_t)n);
        e.launches += 1;
    } else {
        cudaMemsetAsync(w->d_obs + 3 * (size_t)n, 0, sizeof(double) * n, e.st);
    }
    cudaEventRecord(w->ev[4], e.st);
    if (corr_bins > 0) {
        const size_t need = (size_t)n * 3 * corr_bins * corr_bins;
        if (w->corr_cap < need) {
            if (w->d_corr) cudaFree(w->d_corr);
            w->d_corr = nullptr;
            w->corr_cap = 0;
            if (cudaMalloc(&w->d_corr, sizeof(double) * need) != cudaSuccess) {
                e.err = "eigenvalue analysis: correlation matrices allocation failed";
                return SDDDST_ERR_NOMEM;
            }
            w->corr_cap = need;
        }
        if (!w->d_code && cudaMalloc(&w->d_code, sizeof(int) * nn) != cudaSuccess) {
            e.err = "eigenvalue analysis: pair codes allocation failed";
            return SDDDST_ERR_NOMEM;
        }
        pair_code_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, e.st>>>(n, corr_bins, x, e.d_y, e.d_b, w->d_code);
        const size_t smem = sizeof(double) * 2 * corr_bins * corr_bins;
        if (smem <= 200 * 1024) {
            cudaFuncSetAttribute(correl_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            correl_kernel<true><<<n, 512, smem, e.st>>>(n, corr_bins, w->d_H, w->d_code, w->d_corr);
        } else {
            cudaMemsetAsync(w->d_corr, 0, sizeof(double) * need, e.st);
            correl_kernel<false><<<n, 512, 0, e.st>>>(n, corr_bins, w->d_H, w->d_code, w->d_corr);
        }
        e.launches += 2;
    }
    cudaEventRecord(w->ev[5], e.st);
    int info = 0;
    cudaMemcpyAsync(&info, w->d_info, sizeof(int), cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("eigenvalue analysis")) return rc;
    if (info != 0) {
        e.err = "eigenvalue analysis: the eigensolver reported info " + std::to_string(info);
        return SDDDST_ERR_SOLVER;
    }
    for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&w->ms[k], w->ev[k], w->ev[k + 1]);
    return 0;
}

const double *ev_vectors(Engine &e) { return static_cast<EvWork *>(e.ev)->d_H; }
const double *ev_values(Engine &e) { return static_cast<EvWork *>(e.ev)->d_w; }
const double *ev_observables(Engine &e) { return static_cast<EvWork *>(e.ev)->d_obs; }
const double *ev_correlations(Engine &e) { return static_cast<EvWork *>(e.ev)->d_corr; }
void ev_timings(Engine &e, double *ms)
{
    EvWork *w = static_cast<EvWork *>(e.ev);
    for (int k = 0; k < 5; ++k) ms[k] = w ? w->ms[k] : 0.0;
}

} // namespace sd
