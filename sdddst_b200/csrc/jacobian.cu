// Cutoff-sparse Jacobian assembled straight into CSR on the device
// (reference: Simulation::calculateJacobian, src/simulation.cpp:236-384).
//
// The reference scans all N^2/2 pairs on the host and keeps those with
// (r - c)^2 < 36.8 c^2, i.e. r < (1 + sqrt(36.8)) c; here a cell list with
// cells no smaller than that radius limits the scan to the 3x3 neighbouring
// cells.  The matrix kept is the unit-step part G = H/h of
//   J(h) = I + diag((1 + d)/2) h G,
//   G_ij = b_i b_j dtau/dx(dx, dy) w(r)   (i != j),  w = 1 for r <= c,
//                                          exp(-(r-c)^2/c^2) beyond,
//   G_ii = -(sum_j G_ij + sum_defects b_i dF/dx w)        (:269-363),
//   d_i  = (s/(1+s))^2 for s = h G_ii > 0, else 0          (:363-373),
// one CSR row per dislocation with the diagonal in the row's first slot.
// Pair values are evaluated with dx = x[max(i,j)] - x[min(i,j)] as the
// reference does (its rows above the diagonal are copies), so G is exactly
// symmetric.
#include "engine.h"
#include "field_f64.cuh"
#include "field_f32.cuh"
#include "tabulated_field.cuh"

namespace sd {

__device__ __forceinline__ int cell_of(double v, int G)
{
    double w = wrap_half(v) + 0.5;
    int c = (int)floor(w * (double)G);
    return c < 0 ? 0 : (c >= G ? G - 1 : c);
}

__global__ void cell_assign_kernel(int n, const double *__restrict__ x, const double *__restrict__ y, int G,
                                   int *__restrict__ cell, int *__restrict__ count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cell_of(y[i], G) * G + cell_of(x[i], G);
    cell[i] = c;
    atomicAdd(&count[c], 1);
}

// Exclusive scan of m ints by one block: out[0] = 0, out[k+1] = sum_{<=k}.
// Tiles of 512 consecutive elements per warp (16 rounds of 32): each round
// is loaded and stored lane-consecutive (coalesced; all sixteen loads are in
// flight together) and scanned with shuffles, the round's total carried to
// the next; one warp then scans the warp totals (two barriers per tile of
// blockDim.x * 16 elements).  Sums run in 64 bits.
__global__ void scan_kernel(const int *__restrict__ in, int m, int *__restrict__ out)
{
    constexpr int R = 16;
    __shared__ long long warp_tot[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    long long carry = 0;
    for (int base = 0; base < m; base += blockDim.x * R) {
        const int w0 = base + wid * 32 * R;
        int v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = w0 + r * 32 + lane;
            v[r] = k < m ? in[k] : 0;
        }
        long long pre[R];
        long long run = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            long long s = v[r];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += t;
            }
            pre[r] = run + s;
            run += __shfl_sync(0xffffffffu, s, 31);
        }
        if (lane == 0) warp_tot[wid] = run;
        __syncthreads();
        if (wid == 0) {
            long long t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long u = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += u;
            }
            if (lane < nw) warp_tot[lane] = t;
        }
        __syncthreads();
        const long long off = carry + (wid > 0 ? warp_tot[wid - 1] : 0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = w0 + r * 32 + lane;
            if (k < m) out[k + 1] = (int)(off + pre[r]);
        }
        carry += warp_tot[nw - 1];
        __syncthreads(); // warp_tot is rewritten by the next tile
    }
    if (tid == 0) out[0] = 0;
}

// Chunk pass of the multi-block scan: block b scans elements [2048 b,
// 2048 b + 2048) (8 warps x 8 rounds of 32, coalesced), writes the chunk's
// inclusive prefixes to out[k + 1] and its total to tot[b].
__global__ void __launch_bounds__(256) scan_chunks_kernel(const int *__restrict__ in, int m, int *__restrict__ out,
                                                          int *__restrict__ tot)
{
    constexpr int R = 8;
    __shared__ int warp_tot[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int w0 = blockIdx.x * 2048 + wid * 32 * R;
    int v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = w0 + r * 32 + lane;
        v[r] = k < m ? in[k] : 0;
    }
    int pre[R];
    int run = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        int s = v[r];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        pre[r] = run + s;
        run += __shfl_sync(0xffffffffu, s, 31);
    }
    if (lane == 0) warp_tot[wid] = run;
    __syncthreads();
    int off = 0;
    for (int q = 0; q < wid; ++q) off += warp_tot[q];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = w0 + r * 32 + lane;
        if (k < m) out[k + 1] = off + pre[r];
    }
    if (threadIdx.x == 0) {
        int t = 0;
        for (int q = 0; q < 8; ++q) t += warp_tot[q];
        tot[blockIdx.x] = t;
    }
}

// One-launch multi-block scan for up to kOnePassChunks chunks: block b first
// sums everything before its chunk itself (int4 loads; at most 63 x 2048
// entries re-read, 0.5 MB), then scans its chunk as the chunk pass does and
// writes the finished prefixes.  No block waits for another.
constexpr int kOnePassChunks = 64;

__global__ void __launch_bounds__(256) scan_onepass_kernel(const int *__restrict__ in, int m, int *__restrict__ out)
{
    constexpr int R = 8;
    __shared__ int warp_tot[8], warp_pre[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int lim = blockIdx.x * 2048;
    int s = 0;
    if ((reinterpret_cast<size_t>(in) & 15) == 0) {
        const int4 *in4 = reinterpret_cast<const int4 *>(in);
        for (int k = threadIdx.x; k < lim / 4; k += blockDim.x) {
            const int4 v = in4[k];
            s += v.x + v.y + v.z + v.w;
        }
    } else {
        for (int k = threadIdx.x; k < lim; k += blockDim.x) s += in[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) warp_pre[wid] = s;
    const int w0 = lim + wid * 32 * R;
    int v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = w0 + r * 32 + lane;
        v[r] = k < m ? in[k] : 0;
    }
    int pre[R];
    int run = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        int t = v[r];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        pre[r] = run + t;
        run += __shfl_sync(0xffffffffu, t, 31);
    }
    if (lane == 0) warp_tot[wid] = run;
    __syncthreads();
    int off = 0;
    for (int q = 0; q < 8; ++q) off += warp_pre[q];
    for (int q = 0; q < wid; ++q) off += warp_tot[q];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = w0 + r * 32 + lane;
        if (k < m) out[k + 1] = off + pre[r];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0;
}

// Add pass: out[k + 1] += offs[b] over chunk b; out[0] = 0.
__global__ void scan_add_kernel(int m, int *__restrict__ out, const int *__restrict__ offs)
{
    const int b = blockIdx.x;
    const int add = offs[b];
    for (int k = b * 2048 + threadIdx.x; k < min(m, (b + 1) * 2048); k += blockDim.x) out[k + 1] += add;
    if (b == 0 && threadIdx.x == 0) out[0] = 0;
}

// Exclusive scan of m ints: one block up to 2048 entries; up to 64 chunks of
// 2048, one launch in which every block adds up its own prefix; above,
// chunks of 2048 scanned by one block each, their totals scanned by one
// block, and the offsets added (the engine's scan scratch holds totals and
// offsets).  One
// block alone is bound by its load and store round trips (about 22 us for
// 32768 entries).  The output is int32 on both routes, so the total must fit
// in an int: the one-block route sums in 64 bits and narrows on the store,
// the chunked route sums in 32 bits; they agree whenever the total fits.  The
// callers stay far below 2^31: a CSR total is at most N^2 (below 2^31 for
// N <= 46340; N (1 + k) = 2.1e7 at N = 32768, k = 627) and the
// preconditioner's pattern counts are below 32 N.
int launch_scan(Engine &e, const int *in, int m, int *out, cudaStream_t st)
{
    const int nb = (m + 2047) / 2048;
    if (m <= 2048) {
        scan_kernel<<<1, 1024, 0, st>>>(in, m, out);
        return 1;
    }
    if (nb <= kOnePassChunks) {
        scan_onepass_kernel<<<nb, 256, 0, st>>>(in, m, out);
        return 1;
    }
    if (!e.d_scan_tmp || 2 * nb + 2 > e.scan_tmp_cap) {
        scan_kernel<<<1, 1024, 0, st>>>(in, m, out);
        return 1;
    }
    int *tot = e.d_scan_tmp, *offs = e.d_scan_tmp + nb + 1;
    scan_chunks_kernel<<<nb, 256, 0, st>>>(in, m, out, tot);
    scan_kernel<<<1, 1024, 0, st>>>(tot, nb, offs);
    scan_add_kernel<<<nb, 256, 0, st>>>(m, out, offs);
    return 3;
}

__global__ void cell_scatter_kernel(int n, const int *__restrict__ cell, const int *__restrict__ start,
                                    int *__restrict__ fill, int *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cell[i];
    int pos = start[c] + atomicAdd(&fill[c], 1);
    out[pos] = i;
}

// One block per cell: rank sort of the cell's indices (ascending), so the
// neighbour enumeration order never depends on atomic arrival order.
__global__ void cell_sort_kernel(const int *__restrict__ start, const int *__restrict__ in, int *__restrict__ out)
{
    const int c = blockIdx.x;
    const int s = start[c], e = start[c + 1], len = e - s;
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
        int v = in[s + k];
        int rank = 0;
        for (int q = 0; q < len; ++q) rank += in[s + q] < v;
        out[s + rank] = v;
    }
}

struct CellScan {
    int G;
    const int *start;
    const int *sorted;
    const double *xs, *ys; // positions in the cell-sorted order (contiguous per cell)
    double keep_below, keep_above; // r^2 bounds of the cheap decision (see pair_kept_search)
    float kb_f, ka_f;              // the same from FP32 copies of the positions, with a wider margin
};

// Minimum-image difference in FP32 for positions already wrapped into
// [-0.5, 0.5): d - rint(d) with rint as the add/subtract of 1.5 * 2^23.
__device__ __forceinline__ float wrap_diff_f32(float d)
{
    const float m = 12582912.0f;
    return d - __fadd_rn(__fadd_rn(d, m), -m);
}

// Minimum-image difference in FP64 (branch-free; |d| < 2^51): the same value
// as wrap_half except at exactly +1/2, which it keeps.
__device__ __forceinline__ double wrap_diff_f64(double d)
{
    const double m = 6755399441055744.0;
    return d - __dadd_rn(__dadd_rn(d, m), -m);
}

// Visits the cells around (cx, cy) once each: 3x3 for G >= 3, all cells
// otherwise.
template <typename F>
__device__ __forceinline__ void for_neighbour_cells(int cx, int cy, int G, F &&f)
{
    if (G < 3) {
        for (int c = 0; c < G * G; ++c) f(c);
        return;
    }
    for (int oy = -1; oy <= 1; ++oy) {
        int yy = cy + oy;
        yy = yy < 0 ? yy + G : (yy >= G ? yy - G : yy);
        for (int ox = -1; ox <= 1; ++ox) {
            int xx = cx + ox;
            xx = xx < 0 ? xx + G : (xx >= G ? xx - G : xx);
            f(yy * G + xx);
        }
    }
}

// (sqrt(r^2) - c)^2 < 36.8 c^2 and the weight exp(-(r - c)^2 / c^2) beyond c
// (simulation.cpp:335-341), with the reference's roundings (no FMA).
__device__ __forceinline__ bool pair_kept(double r2, double c, double c2, double ic2, double *w_out)
{
    double t = __dsub_rn(sqrt(r2), c);
    double t2 = __dmul_rn(t, t);
    bool keep = t2 < __dmul_rn(36.8, c2);
    if (w_out) *w_out = (r2 > c2) ? exp(__dmul_rn(-t2, ic2)) : 1.0;
    return keep;
}

// pair_kept without its weight, for the neighbour search: r^2 more than 1e-6
// (relative) inside or outside the pattern radius (1 + sqrt(36.8)) c is
// decided without the square root; only the thin shell between takes the
// reference's rounded test, so every decision equals pair_kept's.
__device__ __forceinline__ bool pair_kept_search(double r2, double c, double c2, double ic2, const CellScan &cs)
{
    if (r2 < cs.keep_below) return true;
    if (r2 > cs.keep_above) return false;
    return pair_kept(r2, c, c2, ic2, nullptr);
}

__global__ void gather_cells_kernel(int n, const int *__restrict__ sorted, const double *__restrict__ x,
                                    const double *__restrict__ y, const double *__restrict__ b,
                                    double *__restrict__ xs, double *__restrict__ ys, double *__restrict__ bs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int j = sorted[k];
    xs[k] = x[j];
    ys[k] = y[j];
    bs[k] = b[j];
}

// Candidate test of row i against candidate j at (xj, yj): the reference's
// pattern rule with dx = x[hi] - x[lo].
__device__ __forceinline__ bool cand_kept(int i, double xi, double yi, int j, double xj, double yj, double c,
                                          double c2, double ic2, const CellScan &cs)
{
    const double dx = wrap_half(i < j ? xj - xi : xi - xj);
    const double dy = wrap_half(i < j ? yj - yi : yi - yj);
    return pair_kept_search(r2_exact(dx, dy), c, c2, ic2, cs);
}

// Pattern entries of row i (diagonal excluded), candidates read from global
// memory cell by cell (the fallback when a cell's 3x3 block does not fit in
// shared memory).
__device__ int row_count_global(int i, double xi, double yi, const CellScan &cs, double c, double c2, double ic2,
                                int lane)
{
    const int cx = cell_of(xi, cs.G), cy = cell_of(yi, cs.G);
    int cnt = 0;
    for_neighbour_cells(cx, cy, cs.G, [&](int cell) {
        const int s = cs.start[cell], e = cs.start[cell + 1];
        for (int k = s + lane; k < e; k += 32) {
            const int j = cs.sorted[k];
            if (j != i) cnt += cand_kept(i, xi, yi, j, cs.xs[k], cs.ys[k], c, c2, ic2, cs);
        }
    });
    return cnt;
}

// Columns of row i in cell order, ascending index inside a cell; returns the
// next free slot (rowend when the count pass agreed).
__device__ int row_cols_global(int i, double xi, double yi, const CellScan &cs, double c, double c2, double ic2,
                               int pos, int rowend, int *col, int *col_s, unsigned short *col_s16, int lane)
{
    const int cx = cell_of(xi, cs.G), cy = cell_of(yi, cs.G);
    for_neighbour_cells(cx, cy, cs.G, [&](int cell) {
        const int s = cs.start[cell], e = cs.start[cell + 1];
        for (int k0 = s; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            bool hit = false;
            int j = -1;
            if (k < e) {
                j = cs.sorted[k];
                if (j != i) hit = cand_kept(i, xi, yi, j, cs.xs[k], cs.ys[k], c, c2, ic2, cs);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int at = pos + __popc(m & ((1u << lane) - 1u));
            if (hit && at < rowend) {
                col[at] = j;
                col_s[at] = k; // position of j in the cell-sorted order
                if (col_s16) col_s16[at] = (unsigned short)k;
            }
            pos += __popc(m);
        }
    });
    return pos;
}

// Values of row i (all lanes busy) and its diagonal: G_ij for the columns
// already in place, the point-defect seed (simulation.cpp:274-325), and
// G_ii = -(row sum + defect sum) in the row's first slot.
template <typename VT>
__device__ void row_values(int i, double xi, double yi, double bi, const CellScan &cs, double c, double c2,
                           double ic2, int base, int end, int *col, const int *col_s, VT *val, double *gdiag, int p,
                           const double *pdx, const double *pdy, double A, double K, const double *tab_dx,
                           const double *bs, int lane)
{
    double rs = 0.0;
    if (sizeof(VT) == sizeof(float) && !tab_dx) {
        // FP32 values: two entries per lane (q and q + 32) through the packed field
        for (int qa = base + 1 + lane; qa < end; qa += 64) {
            const int qb = qa + 32;
            const bool hb = qb < end;
            double dxs[2], dys[2], ws[2], bss[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int q = u ? qb : qa;
                if (u && !hb) { // a stand-in pair, never stored
                    dxs[u] = dys[u] = 0.25;
                    ws[u] = bss[u] = 0.0;
                    continue;
                }
                const int j = col[q], ks = col_s[q];
                const double xj = cs.xs[ks], yj = cs.ys[ks];
                dxs[u] = wrap_diff_f64(i < j ? xj - xi : xi - xj); // x[hi] - x[lo]
                dys[u] = wrap_diff_f64(i < j ? yj - yi : yi - yj);
                const double r2 = r2_exact(dxs[u], dys[u]);
                float wf = 1.0f;
                if (r2 > c2) { // the weight of an FP32 value: r from the FP32 reciprocal square root
                    const float r2f = (float)r2;
                    const float t = r2f * rsqrtf(r2f) - (float)c;
                    wf = __expf(-(t * t) * (float)ic2);
                }
                ws[u] = (double)wf;
                bss[u] = bs[ks];
            }
            const float2 t = tau_xy_dx_f32x2(make_float2(__double2float_rn(dxs[0]), __double2float_rn(dxs[1])),
                                             make_float2(__double2float_rn(dys[0]), __double2float_rn(dys[1])));
            // b_i b_j is +-1 (0 for a stand-in): the product runs in FP32, the
            // precision it is stored in, and is the same from either row
            const VT va = (VT)((float)(bi * bss[0]) * (t.x * (float)ws[0]));
            val[qa] = va;
            rs += (double)va;
            if (hb) {
                const VT vb = (VT)((float)(bi * bss[1]) * (t.y * (float)ws[1]));
                val[qb] = vb;
                rs += (double)vb;
            }
        }
    } else {
        for (int q = base + 1 + lane; q < end; q += 32) {
            const int j = col[q], ks = col_s[q];
            const double xj = cs.xs[ks], yj = cs.ys[ks];
            const double ddx = i < j ? xj - xi : xi - xj, ddy = i < j ? yj - yi : yi - yj; // x[hi] - x[lo]
            // FP64 values keep the reference's wrap; FP32 values take the branch-free one
            const double dx = sizeof(VT) == sizeof(double) ? wrap_half(ddx) : wrap_diff_f64(ddx);
            const double dy = sizeof(VT) == sizeof(double) ? wrap_half(ddy) : wrap_diff_f64(ddy);
            double w, tdx;
            if (sizeof(VT) == sizeof(double)) {
                pair_kept(r2_exact(dx, dy), c, c2, ic2, &w);
            } else { // the value is stored in FP32: its weight needs no FP64 square root and exponential
                const double r2 = r2_exact(dx, dy);
                float wf = 1.0f;
                if (r2 > c2) {
                    const float t = sqrtf((float)r2) - (float)c;
                    wf = __expf(-(t * t) * (float)ic2);
                }
                w = (double)wf;
            }
            if (tab_dx) tdx = tau0_xy_dx(dx, dy) + tab_interp(tab_dx, dx, dy); // tabulated field
            else if (sizeof(VT) == sizeof(double)) tdx = tau_xy_dx_f64(dx, dy);
            else tdx = (double)tau_xy_dx_f32(__double2float_rn(dx), __double2float_rn(dy));
            const VT v = (VT)(bi * bs[ks] * tdx * w);
            val[q] = v;
            rs += (double)v;
        }
    }
    double pd = 0.0;
    for (int q = lane; q < p; q += 32) {
        double dx = wrap_half(xi - pdx[q]);
        double dy = wrap_half(yi - pdy[q]);
        double w;
        if (pair_kept(r2_exact(dx, dy), c, c2, ic2, &w)) pd += bi * pd_force_dx_f64(dx, dy, A, K) * w;
    }
    rs = warp_sum(rs);
    pd = warp_sum(pd);
    if (lane == 0) {
        col[base] = i;
        val[base] = (VT)(-(rs + pd));
        gdiag[i] = -(rs + pd);
    }
}

// Count (kFill = false) or fill (kFill = true) pass over the rows of one
// cell.  Block (cell, part) stages the cell's 3x3 neighbour block (FP32
// copies of the wrapped positions and the indices of up to kCandCap
// candidates, in visiting order) in shared memory once; its warps then test
// their rows against it, one row per warp at a time, the cell's rows split
// into `parts` contiguous ranges.  The FP32 r^2 decides every candidate
// farther than the FP32 error (a relative margin of max(1e-4, 1e-5 / r_p) in
// r^2, well above the 2e-7 (|dx| + |dy|) absolute error of the FP32 r^2)
// from the pattern radius; candidates inside that shell take the reference's
// rounded FP64 test on the FP64 positions.  The row's own entry is the
// candidate at its own position in the centre cell.  A block larger than
// kCandCap (or a grid below 3x3 cells) walks global memory cell by cell with
// the FP64 test instead.  Both routes visit candidates in the same order and
// make the same decisions, so the CSR is the same either way.
constexpr int kCandCap = 4096;
constexpr int kCellThreads = 256;
constexpr size_t kCellSmem = (size_t)kCandCap * (2 * sizeof(float) + sizeof(int));

// Sorted position of staged candidate t (segment search over the <= 9 cells).
__device__ __forceinline__ int cand_pos(int t, const int *seg_start, const int *seg_off)
{
    int sg = 0;
    while (t >= seg_off[sg + 1]) ++sg;
    return seg_start[sg] + (t - seg_off[sg]);
}

// Staged decision for candidate t of row i: FP32 r^2 away from the pattern
// radius, the FP64 test inside the shell.
__device__ __forceinline__ bool staged_kept(int i, double xi, double yi, float xif, float yif, int t,
                                            const float *sxc, const float *syc, const int *sjc,
                                            const int *seg_start, const int *seg_off, double c, double c2,
                                            double ic2, const CellScan &cs)
{
    const float dx = wrap_diff_f32(sxc[t] - xif), dy = wrap_diff_f32(syc[t] - yif);
    const float r2f = fmaf(dx, dx, dy * dy);
    if (r2f < cs.kb_f) return true;
    if (r2f > cs.ka_f) return false;
    const int k = cand_pos(t, seg_start, seg_off);
    return cand_kept(i, xi, yi, sjc[t], cs.xs[k], cs.ys[k], c, c2, ic2, cs);
}

template <bool kFill, typename VT>
__global__ void __launch_bounds__(kCellThreads) cell_rows_kernel(
    int parts, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ b, CellScan cs,
    double c, double c2, double ic2, int *__restrict__ rowcnt, const int *__restrict__ rowptr, int *__restrict__ col,
    VT *__restrict__ val, double *__restrict__ gdiag, int p, const double *__restrict__ pdx,
    const double *__restrict__ pdy, double A, double K, int *__restrict__ flag, const double *__restrict__ tab_dx,
    int *__restrict__ col_s, unsigned short *__restrict__ col_s16, const double *__restrict__ bs, long cap)
{
    extern __shared__ __align__(16) unsigned char cell_smem[];
    float *sxc = reinterpret_cast<float *>(cell_smem);
    float *syc = sxc + kCandCap;
    int *sjc = reinterpret_cast<int *>(syc + kCandCap);
    __shared__ int seg_start[9], seg_off[10];

    const int G = cs.G;
    const int cell = blockIdx.x / parts, part = blockIdx.x % parts;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int r0 = cs.start[cell], r1 = cs.start[cell + 1];
    const int chunk = (r1 - r0 + parts - 1) / parts;
    const int rbeg = r0 + part * chunk, rend = min(r0 + (part + 1) * chunk, r1);
    if (rbeg >= rend) return; // whole block: no barrier below is reached

    bool staged = false;
    int ncand = 0;
    if (G >= 3) {
        if (threadIdx.x == 0) {
            const int cx = cell % G, cy = cell / G;
            int nseg = 0, off = 0;
            for_neighbour_cells(cx, cy, G, [&](int nc) {
                seg_start[nseg] = cs.start[nc];
                seg_off[nseg] = off;
                off += cs.start[nc + 1] - cs.start[nc];
                ++nseg;
            });
            seg_off[9] = off;
        }
        __syncthreads();
        ncand = seg_off[9];
        staged = ncand <= kCandCap;
        if (staged) {
            for (int t = threadIdx.x; t < ncand; t += blockDim.x) {
                int sgi = 0;
                while (t >= seg_off[sgi + 1]) ++sgi;
                const int k = seg_start[sgi] + (t - seg_off[sgi]);
                sxc[t] = (float)wrap_half(cs.xs[k]);
                syc[t] = (float)wrap_half(cs.ys[k]);
                sjc[t] = cs.sorted[k];
            }
            __syncthreads();
        }
    }
    for (int r = rbeg + warp; r < rend; r += nwarps) {
        const int i = cs.sorted[r];
        const double xi = x[i], yi = y[i];
        const float xif = (float)wrap_half(xi), yif = (float)wrap_half(yi);
        const int own = staged ? seg_off[4] + (r - seg_start[4]) : -1; // the centre cell is visited fifth
        if (!kFill) {
            int cnt = 0;
            if (staged) {
#pragma unroll 4
                for (int t = lane; t < ncand; t += 32)
                    cnt += t != own &&
                           staged_kept(i, xi, yi, xif, yif, t, sxc, syc, sjc, seg_start, seg_off, c, c2, ic2, cs);
            } else {
                cnt = row_count_global(i, xi, yi, cs, c, c2, ic2, lane);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            if (lane == 0) rowcnt[i] = cnt + 1;
        } else {
            const int base = rowptr[i], rowend = rowptr[i + 1];
            if ((long)rowend > cap) { // the pattern outgrew the CSR storage: report, write nothing
                if (lane == 0) atomicExch(flag, 2);
                continue;
            }
            int pos = base + 1;
            if (staged) {
                int sgi = 0; // segment of the chunk's first candidate (candidates ascend)
                for (int t0 = 0; t0 < ncand; t0 += 32) {
                    const int t = t0 + lane;
                    bool hit = false;
                    if (t < ncand && t != own)
                        hit = staged_kept(i, xi, yi, xif, yif, t, sxc, syc, sjc, seg_start, seg_off, c, c2, ic2,
                                          cs);
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    const int at = pos + __popc(m & ((1u << lane) - 1u));
                    if (hit && at < rowend) {
                        int sg = sgi;
                        while (t >= seg_off[sg + 1]) ++sg;
                        const int k = seg_start[sg] + (t - seg_off[sg]);
                        col[at] = sjc[t];
                        col_s[at] = k;
                        if (col_s16) col_s16[at] = (unsigned short)k;
                    }
                    pos += __popc(m);
                    while (sgi < 8 && t0 + 32 >= seg_off[sgi + 1]) ++sgi;
                }
            } else {
                pos = row_cols_global(i, xi, yi, cs, c, c2, ic2, pos, rowend, col, col_s, col_s16, lane);
            }
            __syncwarp();
            if (pos != rowend) { // count and fill passes disagree: report, never write past the row
                if (lane == 0) atomicExch(flag, 1);
                continue;
            }
            row_values<VT>(i, xi, yi, b[i], cs, c, c2, ic2, base, rowend, col, col_s, val, gdiag, p, pdx, pdy, A, K,
                           tab_dx, bs, lane);
        }
    }
}

// d_i = (s / (1 + s))^2 for s = h G_ii > 0 (simulation.cpp:349-374).
__global__ void make_dvec_kernel(int n, double h, const double *__restrict__ hrow, const double *__restrict__ gdiag,
                                 double *__restrict__ dvec)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = __dmul_rn(hrow ? hrow[i] : h, gdiag[i]);
    double d = 0.0;
    if (s > 0) {
        s = __drcp_rn(s);
        s = __dadd_rn(s, 1.);
        s = __dmul_rn(s, s);
        d = __drcp_rn(s);
    }
    dvec[i] = d;
}

// J values of the CSR (simulation.cpp:376-383): h G_ij (1 + d_i)/2, +1 on the
// diagonal.
template <typename VT>
__global__ void export_j_kernel(int n, double h, const int *__restrict__ rowptr, const VT *__restrict__ val,
                                const double *__restrict__ dvec, double *__restrict__ out)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;
    const double ci = (1.0 + dvec[gw]) * 0.5;
    const int s = rowptr[gw], e = rowptr[gw + 1];
    for (int q = s + lane; q < e; q += 32) {
        double v = h * (double)val[q] * ci;
        out[q] = (q == s) ? v + 1.0 : v;
    }
}

int alloc_csr_values(Engine &e, long cap)
{
    if (e.d_col) cudaFree(e.d_col);
    if (e.d_val) cudaFree(e.d_val);
    if (e.d_valf) cudaFree(e.d_valf);
    e.d_col = nullptr;
    e.d_val = nullptr;
    e.d_valf = nullptr;
    if (cudaMalloc(&e.d_col, sizeof(int) * cap) != cudaSuccess) return SDDDST_ERR_NOMEM;
    if (e.d_col_s) cudaFree(e.d_col_s);
    e.d_col_s = nullptr;
    e.col_s_valid = false;
    if (cudaMalloc(&e.d_col_s, sizeof(int) * cap) != cudaSuccess) return SDDDST_ERR_NOMEM;
    if (e.d_col_s16) cudaFree(e.d_col_s16);
    e.d_col_s16 = nullptr;
    e.col_s16_valid = false;
    if (e.n <= 65536 && !e.batch_backend &&
        cudaMalloc(&e.d_col_s16, sizeof(unsigned short) * cap) != cudaSuccess)
        return SDDDST_ERR_NOMEM;
    if (e.valf) {
        if (cudaMalloc(&e.d_valf, sizeof(float) * cap) != cudaSuccess) return SDDDST_ERR_NOMEM;
    } else {
        if (cudaMalloc(&e.d_val, sizeof(double) * cap) != cudaSuccess) return SDDDST_ERR_NOMEM;
    }
    return 0;
}

static int grow_csr(Engine &e, long need)
{
    if (need <= e.nnz_cap) return 0;
    long cap = need + need / 4 + 1024;
    if (alloc_csr_values(e, cap)) return SDDDST_ERR_NOMEM;
    cudaMemsetAsync(e.d_col, 0, sizeof(int) * cap, e.st);
    e.nnz_cap = cap;
    return 0;
}

// Row ranges per cell for the cell kernels: about three blocks per SM in one
// wave, at least one range per cell.  Sets the kernels' shared-memory limit
// on first use on each device.
static int cell_parts(const Engine &e, int ncell)
{
    static bool attr_set[256] = {};
    const int dev = e.device & 255;
    if (!attr_set[dev]) {
        cudaFuncSetAttribute(cell_rows_kernel<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kCellSmem);
        cudaFuncSetAttribute(cell_rows_kernel<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kCellSmem);
        cudaFuncSetAttribute(cell_rows_kernel<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kCellSmem);
        attr_set[dev] = true;
    }
    const int want = 3 * e.gs_blocks; // gs_blocks: one per SM
    return ncell >= want ? 1 : (want + ncell - 1) / ncell;
}

// With defer, nothing waits for the device: the row counts are not read
// back (the fill is bounded by the current storage and flags an overflow
// with 2 in d_flag) and the fill's flag is left for the caller to read;
// e.nnz is unknown (-1) until then.
int jacobian_assemble(Engine &e, const double *x, bool defer)
{
    const int n = e.n, G = e.G;
    cudaStream_t st = e.st;
    const int ncell = G * G;
    cudaMemsetAsync(e.d_cell_count, 0, sizeof(int) * (ncell + 1), st);
    cudaMemsetAsync(e.d_cell_fill, 0, sizeof(int) * (ncell + 1), st);
    cell_assign_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, e.d_y, G, e.d_cell, e.d_cell_count);
    scan_kernel<<<1, 1024, 0, st>>>(e.d_cell_count, ncell, e.d_cell_start);
    cell_scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, e.d_cell, e.d_cell_start, e.d_cell_fill, e.d_rowcnt);
    cell_sort_kernel<<<ncell, 256, 0, st>>>(e.d_cell_start, e.d_rowcnt, e.d_sorted);
    gather_cells_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, e.d_sorted, x, e.d_y, e.d_b, e.d_xsrt, e.d_ysrt, e.d_bsrt);
    const double rp = e.cutoff * (1.0 + std::sqrt(36.8));
    const double rel = std::max(1e-4, 1e-5 / rp);
    CellScan cs{G, e.d_cell_start, e.d_sorted, e.d_xsrt, e.d_ysrt, rp * rp * (1.0 - 1e-6), rp * rp * (1.0 + 1e-6),
                (float)(rp * rp * (1.0 - rel)), (float)(rp * rp * (1.0 + rel))};
    const int parts = cell_parts(e, ncell);
    const unsigned nb = (unsigned)(ncell * parts);
    cell_rows_kernel<false, float><<<nb, kCellThreads, kCellSmem, st>>>(
        parts, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr, e.d_rowcnt, nullptr, nullptr,
        nullptr, nullptr, 0, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, 0L);
    e.launches += launch_scan(e, e.d_rowcnt, n, e.d_rowptr, st) - 1;
    e.launches += 8;
    if (defer) {
        cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
        if (e.valf)
            cell_rows_kernel<true, float><<<nb, kCellThreads, kCellSmem, st>>>(
                parts, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr, nullptr, e.d_rowptr,
                e.d_col, e.d_valf, e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag, e.d_tab_dx, e.d_col_s,
                e.d_col_s16, e.d_bsrt, e.nnz_cap);
        else
            cell_rows_kernel<true, double><<<nb, kCellThreads, kCellSmem, st>>>(
                parts, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr, nullptr, e.d_rowptr,
                e.d_col, e.d_val, e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag, e.d_tab_dx, e.d_col_s,
                e.d_col_s16, e.d_bsrt, e.nnz_cap);
        e.launches += 1;
        e.nnz = -1;
        e.col_s_valid = true;
        e.col_s16_valid = e.d_col_s16 != nullptr;
        e.spmv_sorted = e.d_sorted;
        return 0;
    }
    int total = 0;
    if (cudaMemcpyAsync(&total, e.d_rowptr + n, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return SDDDST_ERR_CUDA;
    if (int rc = e.sync_check("jacobian count")) return rc;
    if (total < n) {
        e.err = "jacobian: row count overflow";
        return SDDDST_ERR_CAPACITY;
    }
    if (int rc = grow_csr(e, total)) {
        e.err = "jacobian: CSR allocation failed";
        return rc;
    }
    e.nnz = total;
    cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
    if (e.valf)
        cell_rows_kernel<true, float><<<nb, kCellThreads, kCellSmem, st>>>(
            parts, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr, nullptr, e.d_rowptr, e.d_col,
            e.d_valf, e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag, e.d_tab_dx, e.d_col_s, e.d_col_s16,
            e.d_bsrt, e.nnz_cap);
    else
        cell_rows_kernel<true, double><<<nb, kCellThreads, kCellSmem, st>>>(
            parts, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr, nullptr, e.d_rowptr, e.d_col,
            e.d_val, e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag, e.d_tab_dx, e.d_col_s, e.d_col_s16,
            e.d_bsrt, e.nnz_cap);
    e.launches += 1;
    int flag = 0;
    cudaMemcpyAsync(&flag, e.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("jacobian fill")) return rc;
    if (flag) {
        e.err = "jacobian: neighbour count and fill passes disagree";
        return SDDDST_ERR_CAPACITY;
    }
    e.col_s_valid = true;
    e.col_s16_valid = e.d_col_s16 != nullptr;
    e.spmv_sorted = e.d_sorted;
    return 0;
}

// After a deferred fill: stat[0] = entry total of the count pass, stat[1] =
// the fill's flag (1: count and fill disagree, 2: storage overflow); on a
// flag every row pointer is zeroed, so the kernels that follow in the same
// attempt see an empty pattern and read nothing past the storage (the attempt
// is redone on the host's request).  One block.
__global__ void csr_guard_kernel(int n, int *__restrict__ rowptr, const int *__restrict__ flag,
                                 int *__restrict__ stat)
{
    __shared__ int f;
    if (threadIdx.x == 0) {
        f = *flag;
        stat[0] = rowptr[n];
        stat[1] = f;
    }
    __syncthreads();
    if (f != 0)
        for (int i = threadIdx.x; i <= n; i += blockDim.x) rowptr[i] = 0;
}

void launch_csr_guard(Engine &e, int *stat)
{
    csr_guard_kernel<<<1, 256, 0, e.st>>>(e.n, e.d_rowptr, e.d_flag, stat);
    e.launches++;
}

void launch_make_dvec(const Engine &e, double h, double *dvec, cudaStream_t st)
{
    make_dvec_kernel<<<(e.n + 255) / 256, 256, 0, st>>>(e.n, h, e.d_hrow, e.d_gdiag, dvec);
}

void launch_export_jacobian(const Engine &e, double h, const double *dvec, double *val_out, cudaStream_t st)
{
    const int wpb = 8;
    if (e.valf)
        export_j_kernel<float><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(e.n, h, e.d_rowptr, e.d_valf, dvec, val_out);
    else
        export_j_kernel<double><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(e.n, h, e.d_rowptr, e.d_val, dvec, val_out);
}

} // namespace sd
