// Batched stepping of many independent systems of uneven size.
//
// The systems are concatenated into one array of Ntot dislocations
// (system k owns rows off[k] .. off[k+1]-1) and stepped together: every phase
// of the implicit step is one launch over all systems.
//   * pair sum: a tile list (k, I, J) over the systems' own tile triangles,
//     the tile bodies of pair_tile.cuh, per-system partial-sum slabs;
//   * Jacobian: one cell grid per system (its own cutoff c_k = m / sqrt(N_k)
//     and cell count), cells numbered globally; the CSR over all rows is
//     block diagonal by construction;
//   * solve: one cluster-preconditioned GMRES over the block-diagonal union
//     with a per-row step size; each system's right-hand side is scaled to
//     unit norm first, so the union's residual bounds every system's own
//     relative residual by tol sqrt(B);
//   * error ratios, energies and average speeds are segmented reductions
//     (one CTA per system); every system accepts or rejects and adapts its
//     own step size (src/simulation.cpp:501-650 per system).
// The tile size is chosen at creation by timing the pair sum with 32, 64
// and 128 (the autotuner).
//
// After the first step, a step runs with no host round trip and is captured
// once in a CUDA graph, then replayed: the per-system state (step size,
// time, energy, counters, error ratio, speed sums) lives on the device, the
// accept/reject decisions and step-size updates are kernels, the solves are
// the device-resident GMRES, and the assemblies, preconditioner builds and
// solves leave their checks on the device.  One copy after the replay
// brings back the accept flags and the checks; when a check failed (a
// stalled solve, a pattern larger than the CSR storage, a non-finite ratio)
// the step's snapshot is restored and the step is redone by the host-driven
// path, which waits at every check.
#include "engine.h"
#include "pair_tile.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

namespace sd {

struct Batch {
    Engine e; // buffers sized for all rows; e.d_hrow holds per-row step sizes
    int B = 0, T = 64;
    long ntot = 0;
    std::vector<int> nk, off;
    std::vector<long> partoff;
    int *d_inst = nullptr, *d_off = nullptr, *d_tiles = nullptr;
    long ntiles = 0;
    long long *d_partoff = nullptr;
    double *d_bpart = nullptr;
    double *d_hinst = nullptr, *d_cut = nullptr, *d_seg = nullptr, *d_scale = nullptr;
    int *d_G = nullptr, *d_celloff = nullptr, *d_acc = nullptr;
    int *b_cell = nullptr, *b_count = nullptr, *b_start = nullptr, *b_fill = nullptr, *b_sorted = nullptr;
    int ncell_tot = 0;
    // host state per system
    std::vector<double> h, t, energy, ratio, vsq1, vsq2, vsq, avg;
    std::vector<long> succ, failed;
    std::vector<int> accepted;
    bool first = true;
    double *h_seg = nullptr; // pinned, B doubles
    // device-resident stepping: per-system state rows (kState x B doubles),
    // its snapshot and those of x0, v0 and the tolerances, the checks of a
    // step, the captured graph
    double *d_state = nullptr, *d_state_snap = nullptr, *d_x0_snap = nullptr, *d_v0_snap = nullptr;
    double *d_tol_snap = nullptr;
    int *d_check = nullptr;   // [0..2*3) assembly guards, [6..12) preconditioner flags and block counts,
                              // [12] non-finite ratio
    int *h_check = nullptr;   // pinned: checks then accept flags
    bool dev_master = false;  // the device state rows hold the current per-system state
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool graph_failed = false; // capture or instantiation refused: the step is enqueued directly
    long graph_launches = 0;   // kernels one replay launches
    long redone = 0;           // steps redone by the host-driven path
    ~Batch();
};

// rows of Batch::d_state
enum { kSH = 0, kST, kSEnergy, kSRatio, kSVsq1, kSVsq2, kSVsq, kSAvg, kSSucc, kSFailed, kState };

Batch::~Batch()
{
    cudaSetDevice(e.device);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    void *bufs[] = {d_inst, d_off, d_tiles, d_partoff, d_bpart, d_cut, d_seg, d_scale, d_G,
                    d_celloff, d_acc, b_cell, b_count, b_start, b_fill, b_sorted, e.d_hrow, d_state,
                    d_state_snap, d_x0_snap, d_v0_snap, d_tol_snap, d_check};
    for (void *p : bufs)
        if (p) cudaFree(p);
    e.d_hrow = nullptr;
    if (h_seg) cudaFreeHost(h_seg);
    if (h_check) cudaFreeHost(h_check);
}

// ---------------------------------------------------------------- kernels

// only: when not null, systems with only[k] == 0 are skipped (their slabs
// keep their contents)
template <int T, int kMode>
__global__ void __launch_bounds__(T) batch_pair_kernel(const int *__restrict__ tiles, const int *__restrict__ off,
                                                       const long long *__restrict__ partoff,
                                                       const double *__restrict__ x, const double *__restrict__ y,
                                                       const double *__restrict__ b, double *__restrict__ part,
                                                       unsigned long long *__restrict__ minr2, double r2_track,
                                                       const int *__restrict__ only)
{
    const int k = tiles[3 * blockIdx.x], I = tiles[3 * blockIdx.x + 1], J = tiles[3 * blockIdx.x + 2];
    if (only && !only[k]) return;
    const int base = off[k], n = off[k + 1] - base;
    if (kMode == 0)
        pair_tile_f64<T>(x + base, y + base, b + base, n, I, J, part + partoff[k], minr2 + base, r2_track);
    else
        pair_tile_f32<T>(x + base, y + base, b + base, n, I, J, part + partoff[k], minr2 + base, (float)r2_track);
}

__global__ void batch_finish_kernel(long ntot, int T, const int *__restrict__ inst, const int *__restrict__ off,
                                    const long long *__restrict__ partoff, const double *__restrict__ part,
                                    const double *__restrict__ b, double tau_ext, double *__restrict__ S,
                                    double *__restrict__ v, const unsigned long long *__restrict__ minr2,
                                    double *__restrict__ tol, double prec_sqr, int update_tol,
                                    const int *__restrict__ only)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int k = inst[i];
    if (only && !only[k]) return;
    const int base = off[k], n = off[k + 1] - base, il = (int)(i - base);
    const int nblk = (n + T - 1) / T;
    const double *pk = part + partoff[k];
    double acc = 0.0;
    for (int L = 0; L < nblk; ++L) acc += pk[(size_t)L * n + il];
    if (S) S[i] = acc;
    v[i] = acc + b[i] * tau_ext;
    if (update_tol) {
        const double smin = __longlong_as_double((long long)minr2[i]);
        const double t = __dmul_rn(__dmul_rn(smin, 0.25), 1e-2);
        if (t < prec_sqr && t < tol[i]) tol[i] = (t == 0.0) ? kEps : t;
    }
}

__global__ void batch_hrow_kernel(long ntot, const int *__restrict__ inst, const double *__restrict__ hinst,
                                  double factor, double *__restrict__ hrow)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < ntot) hrow[i] = factor * hinst[inst[i]];
}

__device__ __forceinline__ int bcell_of(double v, int G)
{
    double w = wrap_half(v) + 0.5;
    int c = (int)floor(w * (double)G);
    return c < 0 ? 0 : (c >= G ? G - 1 : c);
}

__global__ void batch_cell_assign_kernel(long ntot, const int *__restrict__ inst, const double *__restrict__ x,
                                         const double *__restrict__ y, const int *__restrict__ G,
                                         const int *__restrict__ celloff, int *__restrict__ cell,
                                         int *__restrict__ count)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int k = inst[i], g = G[k];
    const int c = celloff[k] + bcell_of(y[i], g) * g + bcell_of(x[i], g);
    cell[i] = c;
    atomicAdd(&count[c], 1);
}

// shared with speeds.cu and jacobian.cu
__global__ void wrap_kernel(int n, const double *__restrict__ x, double *__restrict__ xw);
__global__ void scan_kernel(const int *__restrict__ in, int m, int *__restrict__ out);
__global__ void cell_scatter_kernel(int n, const int *__restrict__ cell, const int *__restrict__ start,
                                    int *__restrict__ fill, int *__restrict__ out);
__global__ void cell_sort_kernel(const int *__restrict__ start, const int *__restrict__ in, int *__restrict__ out);

__device__ __forceinline__ bool bpair_kept(double r2, double c, double c2, double ic2, double *w_out)
{
    double t = __dsub_rn(sqrt(r2), c);
    double t2 = __dmul_rn(t, t);
    bool keep = t2 < __dmul_rn(36.8, c2);
    if (w_out) *w_out = (r2 > c2) ? exp(__dmul_rn(-t2, ic2)) : 1.0;
    return keep;
}

template <typename F>
__device__ __forceinline__ void batch_cells_around(int k, double xi, double yi, const int *G, const int *celloff,
                                                   F &&f)
{
    const int g = G[k], c0 = celloff[k];
    if (g < 3) {
        for (int c = 0; c < g * g; ++c) f(c0 + c);
        return;
    }
    const int cx = bcell_of(xi, g), cy = bcell_of(yi, g);
    for (int oy = -1; oy <= 1; ++oy) {
        int yy = cy + oy;
        yy = yy < 0 ? yy + g : (yy >= g ? yy - g : yy);
        for (int ox = -1; ox <= 1; ++ox) {
            int xx = cx + ox;
            xx = xx < 0 ? xx + g : (xx >= g ? xx - g : xx);
            f(c0 + yy * g + xx);
        }
    }
}

__global__ void batch_row_count_kernel(long ntot, const int *__restrict__ inst, const double *__restrict__ x,
                                       const double *__restrict__ y, const int *__restrict__ G,
                                       const int *__restrict__ celloff, const double *__restrict__ cut,
                                       const int *__restrict__ start, const int *__restrict__ sorted,
                                       int *__restrict__ rowcnt)
{
    const long gw = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= ntot) return;
    const int i = sorted[gw];
    const int k = inst[i];
    const double c = cut[3 * k], c2 = cut[3 * k + 1], ic2 = cut[3 * k + 2];
    int cnt = 0;
    batch_cells_around(k, x[i], y[i], G, celloff, [&](int cell) {
        for (int q = start[cell] + lane; q < start[cell + 1]; q += 32) {
            const int j = sorted[q];
            if (j == i) continue;
            const int lo = i < j ? i : j, hi = i < j ? j : i;
            double dx = wrap_half(x[hi] - x[lo]), dy = wrap_half(y[hi] - y[lo]);
            cnt += bpair_kept(r2_exact(dx, dy), c, c2, ic2, nullptr);
        }
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) rowcnt[i] = cnt + 1;
}

template <typename VT>
__global__ void batch_row_fill_kernel(long ntot, const int *__restrict__ inst, const double *__restrict__ x,
                                      const double *__restrict__ y, const double *__restrict__ b,
                                      const int *__restrict__ G, const int *__restrict__ celloff,
                                      const double *__restrict__ cut, const int *__restrict__ start,
                                      const int *__restrict__ sorted, const int *__restrict__ rowptr,
                                      int *__restrict__ col, VT *__restrict__ val, double *__restrict__ gdiag,
                                      int *__restrict__ flag, int *__restrict__ col_s, long cap)
{
    const long gw = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= ntot) return;
    const int i = sorted[gw];
    const int k = inst[i];
    const double c = cut[3 * k], c2 = cut[3 * k + 1], ic2 = cut[3 * k + 2];
    const int base = rowptr[i], rowend = rowptr[i + 1];
    if ((long)rowend > cap) { // the pattern outgrew the CSR storage: report, write nothing
        if (lane == 0) atomicExch(flag, 2);
        return;
    }
    int pos = base + 1;
    batch_cells_around(k, x[i], y[i], G, celloff, [&](int cell) {
        const int s = start[cell], e = start[cell + 1];
        for (int k0 = s; k0 < e; k0 += 32) {
            const int q = k0 + lane;
            bool hit = false;
            int j = -1;
            if (q < e) {
                j = sorted[q];
                if (j != i) {
                    const int lo = i < j ? i : j, hi = i < j ? j : i;
                    double dx = wrap_half(x[hi] - x[lo]), dy = wrap_half(y[hi] - y[lo]);
                    hit = bpair_kept(r2_exact(dx, dy), c, c2, ic2, nullptr);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int at = pos + __popc(m & ((1u << lane) - 1u));
            if (hit && at < rowend) {
                col[at] = j;
                col_s[at] = q; // position of j in the sorted list (cell-ordered SpMV gathers)
            }
            pos += __popc(m);
        }
    });
    __syncwarp();
    if (pos != rowend) {
        if (lane == 0) atomicExch(flag, 1);
        return;
    }
    const double bi = b[i];
    double rs = 0.0;
    for (int q = base + 1 + lane; q < rowend; q += 32) {
        const int j = col[q];
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        double dx = wrap_half(x[hi] - x[lo]), dy = wrap_half(y[hi] - y[lo]);
        double w;
        if (sizeof(VT) == sizeof(double)) {
            bpair_kept(r2_exact(dx, dy), c, c2, ic2, &w);
        } else { // FP32 value: FP32 weight
            const double r2 = r2_exact(dx, dy);
            float wf = 1.0f;
            if (r2 > c2) {
                const float t = sqrtf((float)r2) - (float)c;
                wf = __expf(-(t * t) * (float)ic2);
            }
            w = (double)wf;
        }
        double tdx;
        if (sizeof(VT) == sizeof(double)) tdx = tau_xy_dx_f64(dx, dy);
        else tdx = (double)tau_xy_dx_f32(__double2float_rn(dx), __double2float_rn(dy));
        const VT v = (VT)(bi * b[j] * tdx * w);
        val[q] = v;
        rs += (double)v;
    }
    rs = warp_sum(rs);
    if (lane == 0) {
        col[base] = i;
        val[base] = (VT)(-rs);
        gdiag[i] = -rs;
    }
}

// one CTA per system: OP 0 sum a^2, 1 sum |a|, 2 max (a-c)^2/b (error ratio),
// 3 sqrt(sum a^2)
template <int OP>
__global__ void batch_seg_kernel(const int *__restrict__ off, const double *__restrict__ a,
                                 const double *__restrict__ bb, const double *__restrict__ c, double *__restrict__ out)
{
    __shared__ double red[32];
    const int k = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double acc = 0.0;
    for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) {
        double t;
        if (OP == 0 || OP == 3) t = a[i] * a[i];
        else if (OP == 1) t = fabs(a[i]);
        else {
            const double e = fabs(a[i] - c[i]);
            t = e > 0.0 ? __ddiv_rn(__dmul_rn(e, e), bb[i]) : 0.0;
        }
        acc = OP == 2 ? fmax(acc, t) : acc + t;
    }
    acc = OP == 2 ? warp_max(acc) : warp_sum(acc);
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    if (wid == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = OP == 2 ? warp_max(t) : warp_sum(t);
        if (lane == 0) out[k] = OP == 3 ? sqrt(t) : t;
    }
}

__global__ void batch_scale_kernel(long ntot, const int *__restrict__ inst, const double *__restrict__ s,
                                   double *__restrict__ v, int divide)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const double f = s[inst[i]];
    if (f > 0.0) v[i] = divide ? v[i] * f : v[i] / f;
}

__global__ void batch_accept_copy_kernel(long ntot, const int *__restrict__ inst, const int *__restrict__ acc,
                                         const double *__restrict__ src, double *__restrict__ dst)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < ntot && acc[inst[i]]) dst[i] = src[i];
}

// Accept/reject of every system (simulation.cpp:516): acc = ratio < 1; a
// non-finite ratio is reported in check[0].
__global__ void batch_decide_kernel(int B, const double *__restrict__ state, int *__restrict__ acc,
                                    int *__restrict__ check)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B) return;
    const double r = state[kSRatio * B + k];
    if (!isfinite(r)) atomicExch(check, 1);
    acc[k] = r < 1.0 ? 1 : 0;
}

// Bookkeeping of every system after its decision (simulation.cpp:501-650)
// and PrecisionHandler::getNewStepSize (precision_handler.cpp:103-119): time,
// counters, energy, <|v|>, new step size.  avg_sum: sum |v0| at the (new)
// accepted configuration.
__global__ void batch_update_kernel(int B, const int *__restrict__ off, const int *__restrict__ acc,
                                    const double *__restrict__ avg_sum, double *__restrict__ state,
                                    int max_step_limited, double max_step)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B) return;
    double *h = state + kSH * B, *t = state + kST * B, *en = state + kSEnergy * B;
    const double hk = h[k];
    const double vsq1 = state[kSVsq1 * B + k], vsq2 = state[kSVsq2 * B + k], vsq = state[kSVsq * B + k];
    double eacc = (vsq1 + vsq2) * 0.5 * hk * 0.5;
    if (acc[k]) {
        t[k] += hk;
        state[kSSucc * B + k] += 1.0;
        eacc += (vsq2 + vsq) * 0.5 * hk * 0.5;
        en[k] += eacc;
        state[kSAvg * B + k] = avg_sum[k] / double(off[k + 1] - off[k]);
    } else {
        state[kSFailed * B + k] += 1.0;
    }
    const double r = state[kSRatio * B + k];
    double hn;
    if (r == 0.0) hn = 2.0 * hk;
    else hn = 0.9 * hk * fmin(2.0, pow(1. / sqrt(r), 1. / 3.));
    if (max_step_limited && max_step < hn) hn = max_step;
    h[k] = hn;
}

// ------------------------------------------------------------ host side

static unsigned nblocks(long n, int t) { return (unsigned)((n + t - 1) / t); }

static void batch_tiles(Batch &bt, int T, std::vector<int> &tiles, std::vector<long> &partoff)
{
    tiles.clear();
    partoff.assign(bt.B + 1, 0);
    for (int k = 0; k < bt.B; ++k) {
        const int nb = (bt.nk[k] + T - 1) / T;
        for (int J = 0; J < nb; ++J)
            for (int I = 0; I <= J; ++I) {
                tiles.push_back(k);
                tiles.push_back(I);
                tiles.push_back(J);
            }
        partoff[k + 1] = partoff[k] + (long)nb * bt.nk[k];
    }
}

static void launch_batch_pair(Batch &bt, const double *x, double r2_track, const int *only = nullptr)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const int mode = e.prm.pairsum == SDDDST_PAIRSUM_FP32 ? 1 : 0;
    const double *xin = x;
    cudaMemsetAsync(e.d_minr2, 0x7F, sizeof(unsigned long long) * bt.ntot, st); // 0x7F7F.. > any finite r^2
    if (mode == 1) {
        wrap_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>((int)bt.ntot, x, e.d_xw);
        xin = e.d_xw;
        e.launches++;
    }
    const unsigned g = (unsigned)bt.ntiles;
#define SD_BATCH_LAUNCH(TT)                                                                                       \
    if (mode == 0)                                                                                                \
        batch_pair_kernel<TT, 0><<<g, TT, 0, st>>>(bt.d_tiles, bt.d_off, bt.d_partoff, xin, e.d_y, e.d_b,         \
                                                   bt.d_bpart, e.d_minr2, r2_track, only);                        \
    else                                                                                                          \
        batch_pair_kernel<TT, 1><<<g, TT, 0, st>>>(bt.d_tiles, bt.d_off, bt.d_partoff, xin, e.d_y, e.d_b,         \
                                                   bt.d_bpart, e.d_minr2, r2_track, only);
    if (bt.T == 32) {
        SD_BATCH_LAUNCH(32)
    } else if (bt.T == 128) {
        SD_BATCH_LAUNCH(128)
    } else {
        SD_BATCH_LAUNCH(64)
    }
#undef SD_BATCH_LAUNCH
    e.launches++;
}

static void batch_speeds(Batch &bt, const double *x, double *v, double *S, bool update_tol,
                         const int *only = nullptr)
{
    Engine &e = bt.e;
    const double r2_track = update_tol ? 400.0 * e.prec * e.prec * (1.0 + 1e-9) : 0.0;
    launch_batch_pair(bt, x, r2_track, only);
    batch_finish_kernel<<<nblocks(bt.ntot, 256), 256, 0, e.st>>>(bt.ntot, bt.T, bt.d_inst, bt.d_off, bt.d_partoff,
                                                                 bt.d_bpart, e.d_b, 0.0, S, v, e.d_minr2, e.d_tol,
                                                                 e.prec * e.prec, update_tol ? 1 : 0, only);
    e.launches++;
}

static int batch_assemble(Batch &bt, const double *x)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const long n = bt.ntot;
    cudaMemsetAsync(bt.b_count, 0, sizeof(int) * (bt.ncell_tot + 1), st);
    cudaMemsetAsync(bt.b_fill, 0, sizeof(int) * (bt.ncell_tot + 1), st);
    batch_cell_assign_kernel<<<nblocks(n, 256), 256, 0, st>>>(n, bt.d_inst, x, e.d_y, bt.d_G, bt.d_celloff, bt.b_cell,
                                                              bt.b_count);
    scan_kernel<<<1, 1024, 0, st>>>(bt.b_count, bt.ncell_tot, bt.b_start);
    cell_scatter_kernel<<<nblocks(n, 256), 256, 0, st>>>((int)n, bt.b_cell, bt.b_start, bt.b_fill, e.d_rowcnt);
    cell_sort_kernel<<<bt.ncell_tot, 256, 0, st>>>(bt.b_start, e.d_rowcnt, bt.b_sorted);
    batch_row_count_kernel<<<nblocks(n * 32, 256), 256, 0, st>>>(n, bt.d_inst, x, e.d_y, bt.d_G, bt.d_celloff,
                                                                 bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowcnt);
    e.launches += launch_scan(e, e.d_rowcnt, (int)n, e.d_rowptr, st) - 1;
    e.launches += 6;
    int total = 0;
    cudaMemcpyAsync(&total, e.d_rowptr + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("batch jacobian count")) return rc;
    if (total > e.nnz_cap) {
        long cap = total + total / 4 + 1024;
        if (alloc_csr_values(e, cap)) {
            e.err = "batch: CSR allocation failed";
            return SDDDST_ERR_NOMEM;
        }
        cudaMemsetAsync(e.d_col, 0, sizeof(int) * cap, st);
        e.nnz_cap = cap;
    }
    e.nnz = total;
    cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
    if (e.valf)
        batch_row_fill_kernel<float><<<nblocks(n * 32, 256), 256, 0, st>>>(
            n, bt.d_inst, x, e.d_y, e.d_b, bt.d_G, bt.d_celloff, bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowptr,
            e.d_col, e.d_valf, e.d_gdiag, e.d_flag, e.d_col_s, e.nnz_cap);
    else
        batch_row_fill_kernel<double><<<nblocks(n * 32, 256), 256, 0, st>>>(
            n, bt.d_inst, x, e.d_y, e.d_b, bt.d_G, bt.d_celloff, bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowptr,
            e.d_col, e.d_val, e.d_gdiag, e.d_flag, e.d_col_s, e.nnz_cap);
    e.launches++;
    int flag = 0;
    cudaMemcpyAsync(&flag, e.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("batch jacobian fill")) return rc;
    if (flag) {
        e.err = "batch jacobian: count and fill passes disagree";
        return SDDDST_ERR_CAPACITY;
    }
    e.col_s_valid = true;
    e.col_s16_valid = false;
    e.spmv_sorted = bt.b_sorted;
    return 0;
}

static int batch_seg(Batch &bt, int op, const double *a, const double *b, const double *c, std::vector<double> &out)
{
    Engine &e = bt.e;
    switch (op) {
    case 0: batch_seg_kernel<0><<<bt.B, 256, 0, e.st>>>(bt.d_off, a, b, c, bt.d_seg); break;
    case 1: batch_seg_kernel<1><<<bt.B, 256, 0, e.st>>>(bt.d_off, a, b, c, bt.d_seg); break;
    case 2: batch_seg_kernel<2><<<bt.B, 256, 0, e.st>>>(bt.d_off, a, b, c, bt.d_seg); break;
    default: batch_seg_kernel<3><<<bt.B, 256, 0, e.st>>>(bt.d_off, a, b, c, bt.d_seg); break;
    }
    e.launches++;
    cudaMemcpyAsync(bt.h_seg, bt.d_seg, sizeof(double) * bt.B, cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("batch reduction")) return rc;
    out.assign(bt.h_seg, bt.h_seg + bt.B);
    return 0;
}

static void set_hrow(Batch &bt, double factor)
{
    batch_hrow_kernel<<<nblocks(bt.ntot, 256), 256, 0, bt.e.st>>>(bt.ntot, bt.d_inst, bt.d_hinst, factor,
                                                                  bt.e.d_hrow);
    bt.e.launches++;
}

// integrate (simulation.cpp:62-84) for all systems at once; zero external
// stress (the batched workload's loading), so iteration 0 reuses the
// initial velocities.
static int batch_integrate(Batch &bt, double factor, double *xn, const double *xo, bool use2, bool init_speed,
                           bool reuse)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    set_hrow(bt, factor);
    if (!reuse)
        if (int rc = batch_assemble(bt, xn)) return rc;
    launch_make_dvec(e, 0.0, e.d_dvec, st);
    e.launches++;
    if (int rc = e.prepare_solver(0.0)) return rc;
    double *isp = use2 ? e.d_v0b : e.d_v0, *csp0 = use2 ? e.d_vs2 : e.d_vs;
    for (int it = 0; it < e.ic; ++it) {
        if (it == 0 && init_speed) batch_speeds(bt, xo, isp, nullptr, true);
        double *csp = csp0;
        if (it == 0) csp = isp;
        else batch_speeds(bt, xn, csp, nullptr, true);
        launch_residual_g(e, 0.0, xn, xo, csp, isp, e.d_dvec, e.d_g, st);
        // unit-norm right-hand side per system
        batch_seg_kernel<3><<<bt.B, 256, 0, st>>>(bt.d_off, e.d_g, nullptr, nullptr, bt.d_scale);
        batch_scale_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_scale, e.d_g, 0);
        e.launches += 3;
        if (int rc = e.solve(0.0, e.d_g, e.d_sol)) return rc;
        batch_scale_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_scale, e.d_sol, 1);
        launch_axpy_update(e, xn, e.d_sol, st);
        e.launches += 2;
    }
    return 0;
}

static int batch_step_host(Batch &bt, int *accepted_out)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const size_t bytes = sizeof(double) * bt.ntot;
    cudaMemcpyAsync(bt.d_hinst, bt.h.data(), sizeof(double) * bt.B, cudaMemcpyHostToDevice, st);
    if (bt.first) {
        batch_speeds(bt, e.d_x0, e.d_v0, nullptr, true);
        bt.first = false;
    }
    cudaMemcpyAsync(e.d_xb, e.d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate(bt, 1.0, e.d_xb, e.d_x0, false, false, false)) return rc;
    cudaMemcpyAsync(e.d_x1, e.d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate(bt, 0.5, e.d_x1, e.d_x0, false, false, true)) return rc;
    cudaMemcpyAsync(e.d_x2, e.d_x1, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate(bt, 0.5, e.d_x2, e.d_x1, true, true, false)) return rc;
    if (int rc = batch_seg(bt, 0, e.d_v0, nullptr, nullptr, bt.vsq1)) return rc;
    if (int rc = batch_seg(bt, 0, e.d_v0b, nullptr, nullptr, bt.vsq2)) return rc;
    if (int rc = batch_seg(bt, 2, e.d_xb, e.d_tol, e.d_x2, bt.ratio)) return rc;
    int nacc = 0;
    for (int k = 0; k < bt.B; ++k) {
        if (!std::isfinite(bt.ratio[k])) {
            e.err = "batch step: non-finite error ratio";
            return SDDDST_ERR_NONFINITE;
        }
        bt.accepted[k] = bt.ratio[k] < 1.0 ? 1 : 0;
        nacc += bt.accepted[k];
    }
    cudaMemcpyAsync(bt.d_acc, bt.accepted.data(), sizeof(int) * bt.B, cudaMemcpyHostToDevice, st);
    batch_accept_copy_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_acc, e.d_x2, e.d_x0);
    e.launches++;
    std::vector<double> abs_sum(bt.B, 0.0);
    if (nacc > 0) {
        // velocities at the accepted systems' new configurations (the
        // rejected keep x0 and v0)
        batch_speeds(bt, e.d_x0, e.d_v0, nullptr, false, bt.d_acc);
        if (int rc = batch_seg(bt, 0, e.d_v0, nullptr, nullptr, bt.vsq)) return rc;
        if (int rc = batch_seg(bt, 1, e.d_v0, nullptr, nullptr, abs_sum)) return rc;
    }
    for (int k = 0; k < bt.B; ++k) {
        const double hk = bt.h[k];
        double eacc = (bt.vsq1[k] + bt.vsq2[k]) * 0.5 * hk * 0.5;
        if (bt.accepted[k]) {
            bt.t[k] += hk;
            bt.succ[k]++;
            eacc += (bt.vsq2[k] + bt.vsq[k]) * 0.5 * hk * 0.5;
            bt.energy[k] += eacc;
            bt.avg[k] = abs_sum[k] / double(bt.nk[k]);
        } else {
            bt.failed[k]++;
        }
        const double r = bt.ratio[k];
        double hn;
        if (r == 0.0) hn = 2.0 * hk;
        else hn = 0.9 * hk * std::min(2.0, std::pow(1. / std::sqrt(r), 1. / 3.));
        if (e.prm.max_step_limited && e.prm.max_step < hn) hn = e.prm.max_step;
        bt.h[k] = hn;
    }
    // PrecisionHandler::reset for every system
    cudaMemcpyAsync(e.d_tol_last, e.d_tol, bytes, cudaMemcpyDeviceToDevice, st);
    std::vector<double> t0(bt.ntot, e.prec * e.prec);
    cudaMemcpyAsync(e.d_tol, t0.data(), bytes, cudaMemcpyHostToDevice, st);
    if (accepted_out) std::copy(bt.accepted.begin(), bt.accepted.end(), accepted_out);
    return e.sync_check("batch step");
}

// ---- device-resident stepping

// per-system state rows <-> the host vectors of the host-driven path
static void state_to_device(Batch &bt)
{
    const int B = bt.B;
    std::vector<double> st((size_t)kState * B);
    for (int k = 0; k < B; ++k) {
        st[kSH * B + k] = bt.h[k];
        st[kST * B + k] = bt.t[k];
        st[kSEnergy * B + k] = bt.energy[k];
        st[kSRatio * B + k] = bt.ratio[k];
        st[kSVsq1 * B + k] = bt.vsq1[k];
        st[kSVsq2 * B + k] = bt.vsq2[k];
        st[kSVsq * B + k] = bt.vsq[k];
        st[kSAvg * B + k] = bt.avg[k];
        st[kSSucc * B + k] = (double)bt.succ[k];
        st[kSFailed * B + k] = (double)bt.failed[k];
    }
    cudaMemcpyAsync(bt.d_state, st.data(), sizeof(double) * st.size(), cudaMemcpyHostToDevice, bt.e.st);
    cudaStreamSynchronize(bt.e.st);
}

static int state_to_host(Batch &bt)
{
    const int B = bt.B;
    std::vector<double> st((size_t)kState * B);
    cudaMemcpyAsync(st.data(), bt.d_state, sizeof(double) * st.size(), cudaMemcpyDeviceToHost, bt.e.st);
    if (int rc = bt.e.sync_check("batch state")) return rc;
    for (int k = 0; k < B; ++k) {
        bt.h[k] = st[kSH * B + k];
        bt.t[k] = st[kST * B + k];
        bt.energy[k] = st[kSEnergy * B + k];
        bt.ratio[k] = st[kSRatio * B + k];
        bt.vsq1[k] = st[kSVsq1 * B + k];
        bt.vsq2[k] = st[kSVsq2 * B + k];
        bt.vsq[k] = st[kSVsq * B + k];
        bt.avg[k] = st[kSAvg * B + k];
        bt.succ[k] = (long)st[kSSucc * B + k];
        bt.failed[k] = (long)st[kSFailed * B + k];
    }
    return 0;
}

// The assembly without waits: counts, scan, fill bounded by the storage,
// the guard recording the entry total and the fill flag at check[2 slot].
static void batch_assemble_dev(Batch &bt, const double *x, int slot)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const long n = bt.ntot;
    cudaMemsetAsync(bt.b_count, 0, sizeof(int) * (bt.ncell_tot + 1), st);
    cudaMemsetAsync(bt.b_fill, 0, sizeof(int) * (bt.ncell_tot + 1), st);
    batch_cell_assign_kernel<<<nblocks(n, 256), 256, 0, st>>>(n, bt.d_inst, x, e.d_y, bt.d_G, bt.d_celloff, bt.b_cell,
                                                              bt.b_count);
    scan_kernel<<<1, 1024, 0, st>>>(bt.b_count, bt.ncell_tot, bt.b_start);
    cell_scatter_kernel<<<nblocks(n, 256), 256, 0, st>>>((int)n, bt.b_cell, bt.b_start, bt.b_fill, e.d_rowcnt);
    cell_sort_kernel<<<bt.ncell_tot, 256, 0, st>>>(bt.b_start, e.d_rowcnt, bt.b_sorted);
    batch_row_count_kernel<<<nblocks(n * 32, 256), 256, 0, st>>>(n, bt.d_inst, x, e.d_y, bt.d_G, bt.d_celloff,
                                                                 bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowcnt);
    e.launches += launch_scan(e, e.d_rowcnt, (int)n, e.d_rowptr, st) - 1;
    e.launches += 6;
    cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
    if (e.valf)
        batch_row_fill_kernel<float><<<nblocks(n * 32, 256), 256, 0, st>>>(
            n, bt.d_inst, x, e.d_y, e.d_b, bt.d_G, bt.d_celloff, bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowptr,
            e.d_col, e.d_valf, e.d_gdiag, e.d_flag, e.d_col_s, e.nnz_cap);
    else
        batch_row_fill_kernel<double><<<nblocks(n * 32, 256), 256, 0, st>>>(
            n, bt.d_inst, x, e.d_y, e.d_b, bt.d_G, bt.d_celloff, bt.d_cut, bt.b_start, bt.b_sorted, e.d_rowptr,
            e.d_col, e.d_val, e.d_gdiag, e.d_flag, e.d_col_s, e.nnz_cap);
    e.launches++;
    launch_csr_guard(e, bt.d_check + 2 * slot);
    e.col_s_valid = true;
    e.col_s16_valid = false;
    e.spmv_sorted = bt.b_sorted;
}

// batch_integrate without waits: the solves are the device-resident GMRES
// with deferred statuses (slots slot * ic + it), the preconditioner's flag
// and block count go to check[6 + 2 slot].
static int batch_integrate_dev(Batch &bt, double factor, double *xn, const double *xo, bool use2, bool init_speed,
                               bool reuse, int slot)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    set_hrow(bt, factor);
    if (!reuse) batch_assemble_dev(bt, xn, slot);
    launch_make_dvec(e, 0.0, e.d_dvec, st);
    e.launches++;
    if (int rc = precond_build(e, e.pc, 0.0, e.d_dvec, false)) return rc;
    cudaMemcpyAsync(bt.d_check + 6 + 2 * slot, e.pc.flag, sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(bt.d_check + 7 + 2 * slot, e.pc.bbase + bt.ntot, sizeof(int), cudaMemcpyDeviceToDevice, st);
    double *isp = use2 ? e.d_v0b : e.d_v0, *csp0 = use2 ? e.d_vs2 : e.d_vs;
    for (int it = 0; it < e.ic; ++it) {
        if (it == 0 && init_speed) batch_speeds(bt, xo, isp, nullptr, true);
        double *csp = csp0;
        if (it == 0) csp = isp;
        else batch_speeds(bt, xn, csp, nullptr, true);
        launch_residual_g(e, 0.0, xn, xo, csp, isp, e.d_dvec, e.d_g, st);
        batch_seg_kernel<3><<<bt.B, 256, 0, st>>>(bt.d_off, e.d_g, nullptr, nullptr, bt.d_scale);
        batch_scale_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_scale, e.d_g, 0);
        e.launches += 3;
        const double h0 = 0.0;
        const double *dv = e.d_dvec, *rhs = e.d_g;
        double *xs = e.d_sol;
        const Cluster *pcs[1] = {&e.pc};
        if (int rc = fused_gmres(e, 1, &h0, &dv, &rhs, &xs, pcs, nullptr, true, slot * e.ic + it)) return rc;
        batch_scale_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_scale, e.d_sol, 1);
        launch_axpy_update(e, xn, e.d_sol, st);
        e.launches += 2;
    }
    return 0;
}

// One whole step of every system, enqueued with no host round trip (the body
// of the captured graph): snapshot, the three stages, reductions, decisions,
// accepted configurations, their speeds, bookkeeping, tolerance reset.
static int batch_enqueue_step(Batch &bt)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const size_t bytes = sizeof(double) * bt.ntot;
    const int B = bt.B;
    cudaMemcpyAsync(bt.d_state_snap, bt.d_state, sizeof(double) * kState * B, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(bt.d_x0_snap, e.d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(bt.d_v0_snap, e.d_v0, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(bt.d_tol_snap, e.d_tol, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(bt.d_check, 0, sizeof(int) * 16, st);
    cudaMemcpyAsync(e.d_xb, e.d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate_dev(bt, 1.0, e.d_xb, e.d_x0, false, false, false, 0)) return rc;
    cudaMemcpyAsync(e.d_x1, e.d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate_dev(bt, 0.5, e.d_x1, e.d_x0, false, false, true, 1)) return rc;
    cudaMemcpyAsync(e.d_x2, e.d_x1, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = batch_integrate_dev(bt, 0.5, e.d_x2, e.d_x1, true, true, false, 2)) return rc;
    batch_seg_kernel<0><<<B, 256, 0, st>>>(bt.d_off, e.d_v0, nullptr, nullptr, bt.d_state + kSVsq1 * B);
    batch_seg_kernel<0><<<B, 256, 0, st>>>(bt.d_off, e.d_v0b, nullptr, nullptr, bt.d_state + kSVsq2 * B);
    batch_seg_kernel<2><<<B, 256, 0, st>>>(bt.d_off, e.d_xb, e.d_tol, e.d_x2, bt.d_state + kSRatio * B);
    batch_decide_kernel<<<nblocks(B, 128), 128, 0, st>>>(B, bt.d_state, bt.d_acc, bt.d_check + 12);
    batch_accept_copy_kernel<<<nblocks(bt.ntot, 256), 256, 0, st>>>(bt.ntot, bt.d_inst, bt.d_acc, e.d_x2, e.d_x0);
    // speeds at the accepted systems' new configurations (the rejected keep x0 and v0)
    batch_speeds(bt, e.d_x0, e.d_v0, nullptr, false, bt.d_acc);
    batch_seg_kernel<0><<<B, 256, 0, st>>>(bt.d_off, e.d_v0, nullptr, nullptr, bt.d_state + kSVsq * B);
    batch_seg_kernel<1><<<B, 256, 0, st>>>(bt.d_off, e.d_v0, nullptr, nullptr, bt.d_seg);
    batch_update_kernel<<<nblocks(B, 128), 128, 0, st>>>(B, bt.d_off, bt.d_acc, bt.d_seg, bt.d_state,
                                                         e.prm.max_step_limited, e.prm.max_step);
    cudaMemcpyAsync(e.d_tol_last, e.d_tol, bytes, cudaMemcpyDeviceToDevice, st);
    launch_fill(e, e.d_tol, e.prec * e.prec);
    e.launches += 9;
    return 0;
}

// Restores the step's snapshot (per-system state, x0, v0, tolerances).
static void batch_restore(Batch &bt)
{
    Engine &e = bt.e;
    const size_t bytes = sizeof(double) * bt.ntot;
    cudaMemcpyAsync(bt.d_state, bt.d_state_snap, sizeof(double) * kState * bt.B, cudaMemcpyDeviceToDevice, e.st);
    cudaMemcpyAsync(e.d_x0, bt.d_x0_snap, bytes, cudaMemcpyDeviceToDevice, e.st);
    cudaMemcpyAsync(e.d_v0, bt.d_v0_snap, bytes, cudaMemcpyDeviceToDevice, e.st);
    cudaMemcpyAsync(e.d_tol, bt.d_tol_snap, bytes, cudaMemcpyDeviceToDevice, e.st);
}

// One step: the first (and any after a failed check) host-driven; the others
// as a replay of the captured step (or enqueued directly where capture is
// refused), one copy of the checks and accept flags, one wait.
static int batch_step(Batch &bt, int *accepted_out)
{
    Engine &e = bt.e;
    cudaStream_t st = e.st;
    const bool device_path = !bt.first && e.fused && fused_supported(e) && e.ic <= 2;
    if (!device_path) {
        if (bt.dev_master) {
            if (int rc = state_to_host(bt)) return rc;
            bt.dev_master = false;
        }
        return batch_step_host(bt, accepted_out);
    }
    if (!bt.dev_master) {
        state_to_device(bt);
        bt.dev_master = true;
    }
    if (int rc = fused_alloc(e, 1)) {
        e.err = "fused solve: allocation failed";
        return rc;
    }
    if (!bt.gexec && !bt.graph_failed) {
        const long l0 = e.launches;
        bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        int rc = ok ? batch_enqueue_step(bt) : 0;
        cudaGraph_t g = nullptr;
        const bool ended = ok && cudaStreamEndCapture(st, &g) == cudaSuccess && g;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ended && cudaGraphInstantiate(&bt.gexec, g, 0) == cudaSuccess) {
            bt.graph = g;
            bt.graph_launches = e.launches - l0;
            e.launches = l0;
        } else {
            if (g) cudaGraphDestroy(g);
            bt.gexec = nullptr;
            bt.graph_failed = true;
            e.launches = l0;
        }
        (void)cudaGetLastError();
    }
    if (bt.gexec) {
        if (cudaGraphLaunch(bt.gexec, st) != cudaSuccess) {
            e.err = "batch: graph launch failed";
            return SDDDST_ERR_CUDA;
        }
        e.launches += bt.graph_launches;
    } else {
        if (int rc = batch_enqueue_step(bt)) return rc;
    }
    const int B = bt.B;
    cudaMemcpyAsync(bt.h_check, bt.d_check, sizeof(int) * 16, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(bt.h_check + 16, bt.d_acc, sizeof(int) * B, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(e.h_fstatus, e.d_fstatus, sizeof(double) * 4 * 3 * e.ic, cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("batch step")) return rc;
    const int *ck = bt.h_check;
    bool ok = ck[12] == 0;
    int grow = 0;
    for (int a = 0; a < 3; ++a) {
        if (a == 1) continue; // stage II reuses stage I's assembly
        if (ck[2 * a + 1] == 1) {
            e.err = "batch jacobian: count and fill passes disagree";
            return SDDDST_ERR_CAPACITY;
        }
        if (ck[2 * a + 1] == 2) {
            ok = false;
            grow = std::max(grow, ck[2 * a]);
        }
    }
    for (int b = 0; b < 3 && ok; ++b)
        if (ck[6 + 2 * b] != 0 || ck[7 + 2 * b] <= 0 || ck[7 + 2 * b] > bt.ntot) ok = false;
    long its = 0;
    for (int q = 0; q < 3 * e.ic && ok; ++q) {
        const double *sq = e.h_fstatus + 4 * q;
        if (sq[1] == 0.0 || sq[3] != 0.0) ok = false;
        its += (long)sq[0];
    }
    if (!ok) {
        // a deferred check failed: the snapshot back, the step host-driven
        bt.redone++;
        batch_restore(bt);
        if (int rc = state_to_host(bt)) return rc;
        bt.dev_master = false;
        if (grow > 0) { // the storage grows: the captured graph holds the old buffers
            if (bt.gexec) cudaGraphExecDestroy(bt.gexec);
            if (bt.graph) cudaGraphDestroy(bt.graph);
            bt.gexec = nullptr;
            bt.graph = nullptr;
        }
        return batch_step_host(bt, accepted_out);
    }
    e.solves += 3 * e.ic;
    e.iterations += its;
    if (accepted_out) std::copy(bt.h_check + 16, bt.h_check + 16 + B, accepted_out);
    return 0;
}

static double time_pair(Batch &bt, int T)
{
    std::vector<int> tiles;
    std::vector<long> partoff;
    bt.T = T;
    batch_tiles(bt, T, tiles, partoff);
    cudaFree(bt.d_tiles);
    cudaFree(bt.d_partoff);
    cudaFree(bt.d_bpart);
    bt.d_tiles = nullptr;
    bt.d_partoff = nullptr;
    bt.d_bpart = nullptr;
    std::vector<long long> po(partoff.begin(), partoff.end());
    if (cudaMalloc(&bt.d_tiles, sizeof(int) * tiles.size()) != cudaSuccess ||
        cudaMalloc(&bt.d_partoff, sizeof(long long) * po.size()) != cudaSuccess ||
        cudaMalloc(&bt.d_bpart, sizeof(double) * std::max<long>(1, partoff[bt.B])) != cudaSuccess)
        return -1.0;
    cudaMemcpy(bt.d_tiles, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(bt.d_partoff, po.data(), sizeof(long long) * po.size(), cudaMemcpyHostToDevice);
    bt.ntiles = (long)tiles.size() / 3;
    bt.partoff = partoff;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch_batch_pair(bt, bt.e.d_x0, 0.0);
    cudaEventRecord(a, bt.e.st);
    for (int r = 0; r < 3; ++r) launch_batch_pair(bt, bt.e.d_x0, 0.0);
    cudaEventRecord(b, bt.e.st);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / 3.0;
}

static int batch_init(Batch &bt, const sdddst_params &common, int count, const int *sizes, const double *xyb)
{
    bt.B = count;
    bt.nk.assign(sizes, sizes + count);
    bt.off.assign(count + 1, 0);
    for (int k = 0; k < count; ++k) {
        if (sizes[k] < 2) {
            bt.e.err = "batch: every system needs at least 2 dislocations";
            return SDDDST_ERR_INVALID;
        }
        bt.off[k + 1] = bt.off[k] + sizes[k];
    }
    if (common.solver == SDDDST_SOLVER_DIRECT || common.solver == SDDDST_SOLVER_DIRECT_MIXED ||
        common.solver == SDDDST_SOLVER_GMRES_LEARNED ||
        common.solver == SDDDST_SOLVER_GMRES_NEUMANN) {
        bt.e.err = "batch: the sparse LU and learned solvers serve single systems; choose another GMRES solver";
        return SDDDST_ERR_INVALID;
    }
    if (common.field != SDDDST_FIELD_ANALYTIC) {
        bt.e.err = "batch: only the analytic field is supported";
        return SDDDST_ERR_INVALID;
    }
    bt.ntot = bt.off[count];
    if (bt.ntot > (1L << 30)) {
        bt.e.err = "batch too large";
        return SDDDST_ERR_INVALID;
    }
    sdddst_params p = common;
    p.n = (int)bt.ntot;
    p.p = 0;
    p.stress_kind = SDDDST_STRESS_ZERO;
    // one system's cutoff for the engine's bookkeeping; the batch keeps its own per system
    bt.e.batch_backend = true;
    if (int rc = bt.e.init(p, xyb, nullptr)) return rc;
    Engine &e = bt.e;
    const int B = count;
    std::vector<int> inst(bt.ntot), G(B), celloff(B + 1, 0);
    std::vector<double> cut(3 * B);
    for (int k = 0; k < B; ++k) {
        for (int i = bt.off[k]; i < bt.off[k + 1]; ++i) inst[i] = k;
        // SimulationData::updateCutOff per system
        double m = common.cutoff_multiplier;
        if (m >= 1. / 12. * std::sqrt(2.0 * double(bt.nk[k]))) m = 1e20;
        const double c = 1. / std::sqrt((double)bt.nk[k]) * m;
        cut[3 * k] = c;
        cut[3 * k + 1] = c * c;
        cut[3 * k + 2] = 1. / (c * c);
        const double rc = c * (1.0 + std::sqrt(36.8)) * (1.0 + 1e-9);
        int g = rc >= 1.0 / 3.0 ? 1 : (int)std::floor(1.0 / rc);
        if (g < 3) g = 1;
        if (g > 1024) g = 1024;
        G[k] = g;
        celloff[k + 1] = celloff[k] + g * g;
    }
    bt.ncell_tot = celloff[B];
    int rc = 0;
    rc |= cudaMalloc(&bt.d_inst, sizeof(int) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_off, sizeof(int) * (B + 1)) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_state, sizeof(double) * kState * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_state_snap, sizeof(double) * kState * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_x0_snap, sizeof(double) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_v0_snap, sizeof(double) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_tol_snap, sizeof(double) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_check, sizeof(int) * 16) != cudaSuccess;
    rc |= cudaMallocHost(&bt.h_check, sizeof(int) * (16 + B)) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_cut, sizeof(double) * 3 * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_seg, sizeof(double) * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_scale, sizeof(double) * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_G, sizeof(int) * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_celloff, sizeof(int) * (B + 1)) != cudaSuccess;
    rc |= cudaMalloc(&bt.d_acc, sizeof(int) * B) != cudaSuccess;
    rc |= cudaMalloc(&bt.b_cell, sizeof(int) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.b_sorted, sizeof(int) * bt.ntot) != cudaSuccess;
    rc |= cudaMalloc(&bt.b_count, sizeof(int) * (bt.ncell_tot + 1)) != cudaSuccess;
    rc |= cudaMalloc(&bt.b_start, sizeof(int) * (bt.ncell_tot + 1)) != cudaSuccess;
    rc |= cudaMalloc(&bt.b_fill, sizeof(int) * (bt.ncell_tot + 1)) != cudaSuccess;
    rc |= cudaMalloc(&e.d_hrow, sizeof(double) * bt.ntot) != cudaSuccess;
    rc |= cudaMallocHost(&bt.h_seg, sizeof(double) * B) != cudaSuccess;
    if (rc) {
        e.err = "batch: allocation failed";
        return SDDDST_ERR_NOMEM;
    }
    bt.d_hinst = bt.d_state + kSH * B;
    cudaMemcpy(bt.d_inst, inst.data(), sizeof(int) * bt.ntot, cudaMemcpyHostToDevice);
    cudaMemcpy(bt.d_off, bt.off.data(), sizeof(int) * (B + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(bt.d_cut, cut.data(), sizeof(double) * 3 * B, cudaMemcpyHostToDevice);
    cudaMemcpy(bt.d_G, G.data(), sizeof(int) * B, cudaMemcpyHostToDevice);
    cudaMemcpy(bt.d_celloff, celloff.data(), sizeof(int) * (B + 1), cudaMemcpyHostToDevice);
    bt.h.assign(B, common.step_size);
    bt.t.assign(B, 0.0);
    bt.energy.assign(B, 0.0);
    bt.ratio.assign(B, 0.0);
    bt.vsq1.assign(B, 0.0);
    bt.vsq2.assign(B, 0.0);
    bt.vsq.assign(B, 0.0);
    bt.avg.assign(B, 0.0);
    bt.succ.assign(B, 0);
    bt.failed.assign(B, 0);
    bt.accepted.assign(B, 0);
    // autotune the pair-sum tile over {32, 64, 128}
    double best = -1.0;
    int bestT = 64;
    for (int T : {32, 64, 128}) {
        double ms = time_pair(bt, T);
        if (ms > 0 && (best < 0 || ms < best)) {
            best = ms;
            bestT = T;
        }
    }
    if (time_pair(bt, bestT) < 0) {
        e.err = "batch: pair-sum buffers";
        return SDDDST_ERR_NOMEM;
    }
    return e.sync_check("batch init");
}

} // namespace sd

extern "C" {

int sdddst_batch_create(const sdddst_params *common, int count, const int *sizes, const double *xyb, void **batch)
{
    if (!common || !sizes || !xyb || !batch || count < 1) return SDDDST_ERR_INVALID;
    *batch = nullptr;
    long total = 0;
    for (int k = 0; k < count; ++k) total += sizes[k] > 0 ? sizes[k] : 0;
    for (long q = 0; q < 3 * total; ++q)
        if (!std::isfinite(xyb[q])) {
            sd::set_last_error("batch configuration: non-finite value at index " + std::to_string(q));
            return SDDDST_ERR_NONFINITE;
        }
    sd::Batch *bt = new (std::nothrow) sd::Batch();
    if (!bt) return SDDDST_ERR_NOMEM;
    int rc = sd::batch_init(*bt, *common, count, sizes, xyb);
    if (rc) {
        sd::set_last_error(bt->e.err);
        delete bt;
        return rc;
    }
    *batch = bt;
    return SDDDST_OK;
}

int sdddst_batch_destroy(void *batch)
{
    delete static_cast<sd::Batch *>(batch);
    return SDDDST_OK;
}

int sdddst_batch_step(void *batch, int *accepted)
{
    if (!batch) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    cudaSetDevice(bt->e.device);
    int rc = sd::batch_step(*bt, accepted);
    if (rc) sd::set_last_error(bt->e.err);
    return rc;
}

int sdddst_batch_get_scalars(void *batch, double *out)
{
    if (!batch || !out) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    cudaSetDevice(bt->e.device);
    if (bt->dev_master) {
        int rc = sd::state_to_host(*bt);
        if (rc) {
            sd::set_last_error(bt->e.err);
            return rc;
        }
    }
    for (int k = 0; k < bt->B; ++k) {
        double *o = out + 12 * k;
        o[0] = bt->t[k];
        o[1] = bt->h[k];
        o[2] = (double)bt->succ[k];
        o[3] = (double)bt->failed[k];
        o[4] = bt->energy[k];
        o[5] = 0.0;
        o[6] = bt->ratio[k];
        o[7] = bt->avg[k];
        o[8] = bt->vsq[k];
        o[9] = 0.0;
        o[10] = 0.0;
        o[11] = 0.0;
    }
    return SDDDST_OK;
}

int sdddst_batch_get_positions(void *batch, int which, double *x)
{
    if (!batch || !x || which < 0 || which > 3) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    sd::Engine &e = bt->e;
    cudaSetDevice(e.device);
    const double *src = which == 0 ? e.d_x0 : which == 1 ? e.d_xb : which == 2 ? e.d_x1 : e.d_x2;
    cudaMemcpyAsync(x, src, sizeof(double) * bt->ntot, cudaMemcpyDeviceToHost, e.st);
    return e.sync_check("batch positions");
}

int sdddst_batch_profile_pair_sum(void *batch, int reps, double *ms_per_launch, double *pairs)
{
    if (!batch || reps < 1) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    sd::Engine &e = bt->e;
    cudaSetDevice(e.device);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    sd::launch_batch_pair(*bt, e.d_x0, 0.0);
    cudaEventRecord(a, e.st);
    for (int r = 0; r < reps; ++r) sd::launch_batch_pair(*bt, e.d_x0, 0.0);
    cudaEventRecord(b, e.st);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms_per_launch) *ms_per_launch = ms / reps;
    if (pairs) {
        double p = 0;
        for (int k = 0; k < bt->B; ++k) p += 0.5 * (double)bt->nk[k] * (double)(bt->nk[k] - 1);
        *pairs = p;
    }
    return e.sync_check("batch pair profile") ? SDDDST_ERR_CUDA : SDDDST_OK;
}

int sdddst_batch_stats(void *batch, int *graph, long *redone)
{
    if (!batch) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    if (graph) *graph = bt->gexec != nullptr ? 1 : 0;
    if (redone) *redone = bt->redone;
    return SDDDST_OK;
}

int sdddst_batch_info(void *batch, int *tile, long *total, long *launches, void **stream)
{
    if (!batch) return SDDDST_ERR_INVALID;
    sd::Batch *bt = static_cast<sd::Batch *>(batch);
    if (tile) *tile = bt->T;
    if (total) *total = bt->ntot;
    if (launches) *launches = bt->e.launches;
    if (stream) *stream = (void *)bt->e.st;
    return SDDDST_OK;
}

} // extern "C"
