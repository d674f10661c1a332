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
__global__ void scan_kernel(const int *__restrict__ in, int m, int *__restrict__ out)
{
    __shared__ long long warp_tot[32];
    __shared__ long long carry_s;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry_s = 0;
    __syncthreads();
    for (int base = 0; base < m; base += blockDim.x) {
        int k = base + tid;
        long long v = k < m ? in[k] : 0;
        long long s = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane == 31) warp_tot[wid] = s;
        __syncthreads();
        if (wid == 0) {
            int nw = blockDim.x >> 5;
            long long t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                long long u = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += u;
            }
            if (lane < nw) warp_tot[lane] = t;
        }
        __syncthreads();
        long long incl = s + (wid > 0 ? warp_tot[wid - 1] : 0) + carry_s;
        if (k < m) out[k + 1] = (int)incl;
        __syncthreads();
        if (tid == blockDim.x - 1) carry_s = incl;
        __syncthreads();
    }
    if (tid == 0) out[0] = 0;
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
};

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

__global__ void row_count_kernel(int n, const double *__restrict__ x, const double *__restrict__ y, CellScan cs,
                                 double c, double c2, double ic2, int *__restrict__ rowcnt)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;
    const int i = cs.sorted[gw];
    const double xi = x[i], yi = y[i];
    const int cx = cell_of(xi, cs.G), cy = cell_of(yi, cs.G);
    int cnt = 0;
    for_neighbour_cells(cx, cy, cs.G, [&](int cell) {
        const int s = cs.start[cell], e = cs.start[cell + 1];
        for (int k = s + lane; k < e; k += 32) {
            const int j = cs.sorted[k];
            if (j == i) continue;
            const double xj = cs.xs[k], yj = cs.ys[k];
            double dx = wrap_half(i < j ? xj - xi : xi - xj); // x[hi] - x[lo], as the reference orders it
            double dy = wrap_half(i < j ? yj - yi : yi - yj);
            cnt += pair_kept_search(r2_exact(dx, dy), c, c2, ic2, cs);
        }
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) rowcnt[i] = cnt + 1;
}

template <typename VT>
__global__ void row_fill_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ b, CellScan cs, double c, double c2, double ic2,
                                const int *__restrict__ rowptr, int *__restrict__ col, VT *__restrict__ val,
                                double *__restrict__ gdiag, int p, const double *__restrict__ pdx,
                                const double *__restrict__ pdy, double A, double K, int *__restrict__ flag,
                                const double *__restrict__ tab_dx, int *__restrict__ col_s,
                                const double *__restrict__ bs)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;
    const int i = cs.sorted[gw];
    const double xi = x[i], yi = y[i], bi = b[i];
    const int cx = cell_of(xi, cs.G), cy = cell_of(yi, cs.G);
    const int base = rowptr[i];
    const int rowend = rowptr[i + 1];
    int pos = base + 1;
    // 1) columns, in cell order then ascending index inside a cell
    for_neighbour_cells(cx, cy, cs.G, [&](int cell) {
        const int s = cs.start[cell], e = cs.start[cell + 1];
        for (int k0 = s; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            bool hit = false;
            int j = -1;
            if (k < e) {
                j = cs.sorted[k];
                if (j != i) {
                    const double xj = cs.xs[k], yj = cs.ys[k];
                    double dx = wrap_half(i < j ? xj - xi : xi - xj); // x[hi] - x[lo]
                    double dy = wrap_half(i < j ? yj - yi : yi - yj);
                    hit = pair_kept_search(r2_exact(dx, dy), c, c2, ic2, cs);
                }
            }
            unsigned m = __ballot_sync(0xffffffffu, hit);
            const int at = pos + __popc(m & ((1u << lane) - 1u));
            if (hit && at < rowend) {
                col[at] = j;
                col_s[at] = k; // position of j in the cell-sorted order
            }
            pos += __popc(m);
        }
    });
    __syncwarp();
    if (pos != rowend) { // count and fill passes disagree: report, never write past the row
        if (lane == 0) atomicExch(flag, 1);
        return;
    }
    // 2) values, all lanes busy
    const int end = rowend;
    double rs = 0.0;
    for (int q = base + 1 + lane; q < end; q += 32) {
        const int j = col[q], ks = col_s[q];
        const double xj = cs.xs[ks], yj = cs.ys[ks];
        double dx = wrap_half(i < j ? xj - xi : xi - xj); // x[hi] - x[lo]
        double dy = wrap_half(i < j ? yj - yi : yi - yj);
        double w;
        pair_kept(r2_exact(dx, dy), c, c2, ic2, &w);
        double tdx;
        if (tab_dx) tdx = tau0_xy_dx(dx, dy) + tab_interp(tab_dx, dx, dy); // tabulated field
        else if (sizeof(VT) == sizeof(double)) tdx = tau_xy_dx_f64(dx, dy);
        else tdx = (double)tau_xy_dx_f32(__double2float_rn(dx), __double2float_rn(dy));
        const VT v = (VT)(bi * bs[ks] * tdx * w);
        val[q] = v;
        rs += (double)v;
    }
    // 3) point-defect seed of the diagonal (simulation.cpp:274-325)
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

int jacobian_assemble(Engine &e, const double *x)
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
    CellScan cs{G, e.d_cell_start, e.d_sorted, e.d_xsrt, e.d_ysrt, rp * rp * (1.0 - 1e-6), rp * rp * (1.0 + 1e-6)};
    const int wpb = 8; // warps per block
    const unsigned rb = (unsigned)((n + wpb - 1) / wpb);
    row_count_kernel<<<rb, 32 * wpb, 0, st>>>(n, x, e.d_y, cs, e.cutoff, e.cutoff_sqr, e.one_per_cutoff_sqr,
                                              e.d_rowcnt);
    scan_kernel<<<1, 1024, 0, st>>>(e.d_rowcnt, n, e.d_rowptr);
    e.launches += 8;
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
        row_fill_kernel<float><<<rb, 32 * wpb, 0, st>>>(n, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr,
                                                       e.one_per_cutoff_sqr, e.d_rowptr, e.d_col, e.d_valf,
                                                       e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag,
                                                       e.d_tab_dx, e.d_col_s, e.d_bsrt);
    else
        row_fill_kernel<double><<<rb, 32 * wpb, 0, st>>>(n, x, e.d_y, e.d_b, cs, e.cutoff, e.cutoff_sqr,
                                                        e.one_per_cutoff_sqr, e.d_rowptr, e.d_col, e.d_val,
                                                        e.d_gdiag, e.p, e.d_pdx, e.d_pdy, e.A, e.KASQR, e.d_flag,
                                                        e.d_tab_dx, e.d_col_s, e.d_bsrt);
    e.launches += 1;
    int flag = 0;
    cudaMemcpyAsync(&flag, e.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("jacobian fill")) return rc;
    if (flag) {
        e.err = "jacobian: neighbour count and fill passes disagree";
        return SDDDST_ERR_CAPACITY;
    }
    e.col_s_valid = true;
    e.spmv_sorted = e.d_sorted;
    return 0;
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
