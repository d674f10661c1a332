// Cluster block-Jacobi preconditioner for J(h) = I + diag(c) h G,
// c_i = (1 + d_i)/2.
//
// Close dislocation pairs couple through entries of size h |dtau/dx| ~ h/r^2
// that can exceed the identity by orders of magnitude; such a pair forms a
// stiff 2x2 block whose soft mode (both dislocations moving together) a
// diagonal scaling cannot reach.  Strongly coupled dislocations are therefore
// grouped and their diagonal blocks of J inverted exactly:
//   * strength s_ij = h |G_ij| / sqrt(M_ii M_jj) on the symmetric form
//     M = diag(c)^-1 J (M_ii = 1/c_i + h G_ii, M_ij = h G_ij);
//   * every dislocation points to its strongest neighbour with s >= theta;
//     following pointers never decreases s, so each chain ends in a mutual
//     pair, whose smaller index roots the cluster (one bounded walk per
//     dislocation);
//   * clusters are listed contiguously, members in ascending index order,
//     and cut into blocks of at most kMaxBlock;
//   * a one-member block is inverted by one lane; a warp builds each larger
//     block of J densely, inverts it by Gauss-Jordan elimination with
//     partial pivoting in shared memory, and stores the inverse; applying
//     M^-1 is one small dense product per block.
#include "engine.h"
#include "common.cuh"

#include <vector>

namespace sd {

constexpr int kMaxBlock = 32;

// s_ij >= theta  <=>  v^2 / |M_jj| >= theta^2 |M_ii| / h^2  (v = G_ij), and
// within row i the strongest j maximises v^2 / |M_jj|: the search compares
// that key, so a row costs two multiplies per entry instead of a square root
// and a division.  rm_j = 1 / |M_jj| (0 where M_jj = 0: no coupling) comes
// from the cell-sorted copy when present (msrt, read through the CSR's sorted
// column positions, ties broken by the sorted position), else it is formed
// per entry (ties broken by the column index).
template <typename VT>
__global__ void strongest_kernel(int n, double h0, const double *__restrict__ hrow, double theta,
                                 const int *__restrict__ rowptr, const int *__restrict__ col,
                                 const VT *__restrict__ val, const double *__restrict__ gdiag,
                                 const double *__restrict__ dvec, int *__restrict__ ptr,
                                 const int *__restrict__ col_s, const VT *__restrict__ msrt,
                                 const int *__restrict__ sorted)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double h = hrow ? hrow[i] : h0; // couplings never cross systems, so row i's h serves the pair
    const int s = rowptr[i], e = rowptr[i + 1];
    const double mii = 2.0 / (1.0 + dvec[i]) + h * gdiag[i];
    const VT thr = (VT)(theta * theta * fabs(mii) / (h * h));
    VT best = (VT)-1;
    int bid = 0x7fffffff;
    for (int q = s + 1 + lane; q < e; q += 32) {
        const VT v = val[q];
        VT rm;
        int id;
        if (msrt) {
            id = col_s[q];
            rm = msrt[id];
        } else {
            id = col[q];
            const double mjj = 2.0 / (1.0 + dvec[id]) + h * gdiag[id];
            rm = mjj != 0.0 ? (VT)(1.0 / fabs(mjj)) : (VT)0;
        }
        const VT key = v * v * rm;
        if (key >= thr && (key > best || (key == best && id < bid))) {
            best = key;
            bid = id;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const VT ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oid = __shfl_xor_sync(0xffffffffu, bid, o);
        if (ob > best || (ob == best && oid < bid)) {
            best = ob;
            bid = oid;
        }
    }
    if (lane == 0) ptr[i] = best >= thr && bid != 0x7fffffff ? (msrt ? sorted[bid] : bid) : i;
}

// 1 / |M_jj| (M_jj = 2 / (1 + d_j) + h G_jj; 0 where M_jj = 0) in the
// cell-sorted order (single system)
template <typename VT>
__global__ void msorted_kernel(int n, double h, const int *__restrict__ sorted, const double *__restrict__ gdiag,
                               const double *__restrict__ dvec, VT *__restrict__ msrt)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int j = sorted[k];
    const double m = 2.0 / (1.0 + dvec[j]) + h * gdiag[j];
    msrt[k] = m != 0.0 ? (VT)(1.0 / fabs(m)) : (VT)0;
}

// Cluster root of every dislocation in one pass: a dislocation that points
// to itself, or the smaller index of a mutual pair, is a root; every other
// one follows the pointers for at most kRootWalk steps and takes the root it
// reaches, or becomes its own root when none is reached within them (a chain
// longer than that, or a tie cycle).  Roots count their members.
constexpr int kRootWalk = 4096;

__device__ __forceinline__ bool is_root(const int *__restrict__ ptr, int i, int p)
{
    return p == i || (ptr[p] == i && i < p);
}

__global__ void root_walk_kernel(int n, const int *__restrict__ ptr, int *__restrict__ root, int *__restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = i, p = ptr[i];
    int steps = 0;
    while (!is_root(ptr, r, p) && steps < kRootWalk) {
        r = p;
        p = ptr[r];
        ++steps;
    }
    if (!is_root(ptr, r, p)) r = i;
    root[i] = r;
    atomicAdd(&count[r], 1);
}

__global__ void member_scatter_kernel(int n, const int *__restrict__ root, const int *__restrict__ start,
                                      int *__restrict__ fill, int *__restrict__ members)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = root[i];
    members[start[r] + atomicAdd(&fill[r], 1)] = i;
}

// one thread per cluster root: members in ascending order (rank sort, for
// clusters of up to 256; larger ones keep their arrival order) and the
// cluster's block count
__global__ void cluster_sort_kernel(int n, const int *__restrict__ count, const int *__restrict__ start,
                                    const int *__restrict__ in, int *__restrict__ out, int *__restrict__ nblocks)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int k = count[r];
    nblocks[r] = k > 0 ? (k + kMaxBlock - 1) / kMaxBlock : 0;
    if (k == 0) return;
    int s = start[r];
    if (k > 256) {
        for (int a = 0; a < k; ++a) out[s + a] = in[s + a];
        return;
    }
    for (int a = 0; a < k; ++a) {
        int v = in[s + a], rank = 0;
        for (int b2 = 0; b2 < k; ++b2) rank += in[s + b2] < v;
        out[s + rank] = v;
    }
}

__global__ void block_list_kernel(int n, const int *__restrict__ count, const int *__restrict__ start,
                                  const int *__restrict__ bbase, int *__restrict__ bstart, int *__restrict__ blen)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int k = count[r];
    if (k == 0) return;
    int s = start[r], b0 = bbase[r];
    for (int t = 0; t * kMaxBlock < k; ++t) {
        bstart[b0 + t] = s + t * kMaxBlock;
        int len = k - t * kMaxBlock;
        blen[b0 + t] = len < kMaxBlock ? len : kMaxBlock;
    }
}

// nbp: the block count, on the device (no host round trip before the launch)
__global__ void block_meta_kernel(const int *__restrict__ nbp, const int *__restrict__ bstart,
                                  const int *__restrict__ blen, const int *__restrict__ members,
                                  int *__restrict__ blk_of, int *__restrict__ loc, int *__restrict__ sq)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= *nbp) return;
    int s = bstart[b], k = blen[b];
    for (int t = 0; t < k; ++t) {
        int i = members[s + t];
        blk_of[i] = b;
        loc[i] = t;
    }
    sq[b] = k * k;
}

// Dense J block b (k >= 2 members from bstart s), Gauss-Jordan inverse with
// partial pivoting by one warp in M, written row-major at binv[off[b]];
// false when the block is singular.
template <typename VT>
__device__ bool invert_block_warp(int b, int k, int s, double h, const int *__restrict__ members,
                                  const int *__restrict__ blk_of, const int *__restrict__ loc,
                                  const int *__restrict__ off, const int *__restrict__ rowptr,
                                  const int *__restrict__ col, const VT *__restrict__ val,
                                  const double *__restrict__ gdiag, const double *__restrict__ dvec,
                                  double *__restrict__ binv, double (*M)[2 * kMaxBlock + 1], int lane)
{
    for (int r = 0; r < k; ++r)
        for (int c = lane; c < 2 * k; c += 32) M[r][c] = (c - k == r) ? 1.0 : 0.0;
    __syncwarp();
    // gather the block, one member row at a time, the warp scanning the row
    // (the columns of one row are distinct: no two lanes write one entry)
    for (int r = 0; r < k; ++r) {
        const int i = members[s + r];
        const double ci = (1.0 + dvec[i]) * 0.5 * h;
        for (int q = rowptr[i] + 1 + lane; q < rowptr[i + 1]; q += 32) {
            const int j = col[q];
            if (blk_of[j] == b) M[r][loc[j]] += ci * (double)val[q];
        }
        if (lane == 0) M[r][r] += 1.0 + ci * gdiag[i];
        __syncwarp();
    }
    bool singular = false;
    for (int p = 0; p < k; ++p) {
        // pivot search in column p (rows p..k-1)
        double v = lane >= p && lane < k ? fabs(M[lane][p]) : -1.0;
        int idx = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, v, o);
            int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (ov > v || (ov == v && oi < idx)) {
                v = ov;
                idx = oi;
            }
        }
        if (!(v > 0.0)) {
            singular = true;
            break;
        }
        if (idx != p)
            for (int c = lane; c < 2 * k; c += 32) {
                double t = M[p][c];
                M[p][c] = M[idx][c];
                M[idx][c] = t;
            }
        __syncwarp();
        const double inv = 1.0 / M[p][p];
        __syncwarp();
        for (int c = lane; c < 2 * k; c += 32) M[p][c] *= inv;
        __syncwarp();
        if (lane < k && lane != p) {
            const double f = M[lane][p];
            if (f != 0.0)
                for (int c = 0; c < 2 * k; ++c) M[lane][c] -= f * M[p][c];
        }
        __syncwarp();
    }
    if (singular) return false;
    double *dst = binv + off[b];
    for (int r = 0; r < k; ++r)
        for (int c = lane; c < k; c += 32) dst[r * k + c] = M[r][k + c];
    __syncwarp();
    return true;
}

// Each warp serves 32 consecutive blocks: a one-member block (most of them)
// is inverted by its own lane, and the warp then takes the larger blocks
// of its group one after another.
template <typename VT>
__global__ void block_invert_kernel(const int *__restrict__ nbp, double h0, const double *__restrict__ hrow, const int *__restrict__ bstart,
                                    const int *__restrict__ blen,
                                    const int *__restrict__ members, const int *__restrict__ blk_of,
                                    const int *__restrict__ loc, const int *__restrict__ off,
                                    const int *__restrict__ rowptr, const int *__restrict__ col,
                                    const VT *__restrict__ val, const double *__restrict__ gdiag,
                                    const double *__restrict__ dvec, double *__restrict__ binv,
                                    int *__restrict__ flag)
{
    __shared__ double A[2][kMaxBlock][2 * kMaxBlock + 1];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b0 = (blockIdx.x * 2 + wib) * 32;
    const int nb = *nbp;
    if (b0 >= nb) return;
    const int bl = b0 + lane;
    const int kl = bl < nb ? blen[bl] : 0;
    if (kl == 1) {
        const int i = members[bstart[bl]];
        const double h = hrow ? hrow[i] : h0;
        const double jii = 1.0 + (1.0 + dvec[i]) * 0.5 * h * gdiag[i];
        binv[off[bl]] = 1.0 / jii;
    }
    unsigned multi = __ballot_sync(0xffffffffu, kl > 1);
    while (multi) {
        const int l = __ffs(multi) - 1;
        multi &= multi - 1u;
        const int b = b0 + l;
        const int k = blen[b], s = bstart[b];
        const double h = hrow ? hrow[members[s]] : h0; // a block lies inside one system
        if (!invert_block_warp<VT>(b, k, s, h, members, blk_of, loc, off, rowptr, col, val, gdiag, dvec, binv,
                                   A[wib], lane) &&
            lane == 0)
            atomicExch(flag, 1);
    }
}

// z = M^-1 v, one thread per dislocation i: its row loc[i] of its block's
// inverse against the block's members (most blocks hold one or two
// dislocations, so a warp per block would leave most lanes idle).
__global__ void block_apply_kernel(int n, const int *__restrict__ blk_of, const int *__restrict__ loc,
                                   const int *__restrict__ bstart, const int *__restrict__ blen,
                                   const int *__restrict__ members, const int *__restrict__ off,
                                   const double *__restrict__ binv, const double *__restrict__ v,
                                   double *__restrict__ z)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = blk_of[i];
    const int k = blen[b], s = bstart[b];
    const double *B = binv + off[b] + (size_t)loc[i] * k;
    double acc = 0.0;
    for (int c = 0; c < k; ++c) acc += B[c] * v[members[s + c]];
    z[i] = acc;
}

// scan helper from jacobian.cu
__global__ void scan_kernel(const int *__restrict__ in, int m, int *__restrict__ out);

double cluster_theta(const Engine &e)
{
    if (e.prm.precond_theta > 0) return e.prm.precond_theta;
    const bool corrected =
        e.prm.solver == SDDDST_SOLVER_GMRES_LEARNED || e.prm.solver == SDDDST_SOLVER_GMRES_NEUMANN;
    return corrected ? 0.05 : 0.01;
}

// Builds the cluster block-Jacobi inverse of J(h) for the assembled G.
int precond_build(Engine &e, Cluster &c, double h, const double *dvec, bool check)
{
    const int n = e.n;
    cudaStream_t st = e.st;
    const unsigned nb256 = (unsigned)((n + 255) / 256);
    const double theta = cluster_theta(e);
    int *ptr = c.ptr, *par = c.parent;
    // single system: M_jj in the cell-sorted order (the SpMV's staging buffer,
    // free until the solve), read through the CSR's sorted column positions
    const bool srt = e.col_s_valid && !e.d_hrow;
    if (e.valf) {
        float *msrt = srt ? reinterpret_cast<float *>(e.d_vsort) : nullptr;
        if (srt) msorted_kernel<float><<<nb256, 256, 0, st>>>(n, h, e.spmv_sorted, e.d_gdiag, dvec, msrt);
        strongest_kernel<float><<<(n + 7) / 8, 256, 0, st>>>(n, h, e.d_hrow, theta, e.d_rowptr, e.d_col, e.d_valf,
                                                             e.d_gdiag, dvec, ptr, e.d_col_s, msrt, e.spmv_sorted);
    } else {
        double *msrt = srt ? e.d_vsort : nullptr;
        if (srt) msorted_kernel<double><<<nb256, 256, 0, st>>>(n, h, e.spmv_sorted, e.d_gdiag, dvec, msrt);
        strongest_kernel<double><<<(n + 7) / 8, 256, 0, st>>>(n, h, e.d_hrow, theta, e.d_rowptr, e.d_col, e.d_val,
                                                              e.d_gdiag, dvec, ptr, e.d_col_s, msrt, e.spmv_sorted);
    }
    if (srt) e.launches++;
    cudaMemsetAsync(c.count, 0, sizeof(int) * (n + 1), st);
    cudaMemsetAsync(c.fill, 0, sizeof(int) * (n + 1), st);
    root_walk_kernel<<<nb256, 256, 0, st>>>(n, ptr, par, c.count);
    e.launches += launch_scan(e, c.count, n, c.start, st) - 1;
    member_scatter_kernel<<<nb256, 256, 0, st>>>(n, par, c.start, c.fill, c.tmp2);
    cluster_sort_kernel<<<nb256, 256, 0, st>>>(n, c.count, c.start, c.tmp2, c.members, c.nblk);
    e.launches += launch_scan(e, c.nblk, n, c.bbase, st) - 1;
    e.launches += 6;
    // the block count stays on the device (pc_bbase[n]); the block kernels
    // run over n (an upper bound) and return beyond it, and the inverses'
    // storage is sized for the bound sum k^2 <= kMaxBlock n once
    const int *nbp = c.bbase + n;
    const long cap = (long)kMaxBlock * n + 1024;
    if (cap > c.binv_cap) {
        if (c.binv) cudaFree(c.binv);
        c.binv = nullptr;
        c.binv_cap = 0;
        if (cudaMalloc(&c.binv, sizeof(double) * cap) != cudaSuccess) {
            e.err = "precond: allocation failed";
            return SDDDST_ERR_NOMEM;
        }
        c.binv_cap = cap;
    }
    block_list_kernel<<<nb256, 256, 0, st>>>(n, c.count, c.start, c.bbase, c.bstart, c.blen);
    cudaMemsetAsync(c.sq, 0, sizeof(int) * (n + 1), st);
    block_meta_kernel<<<nb256, 256, 0, st>>>(nbp, c.bstart, c.blen, c.members, c.blk_of, c.loc,
                                             c.sq);
    e.launches += launch_scan(e, c.sq, n, c.off, st) - 1;
    cudaMemsetAsync(c.flag, 0, sizeof(int), st);
    const unsigned ib = (unsigned)((n + 63) / 64); // 32 blocks per warp, two warps per CTA
    if (e.valf)
        block_invert_kernel<float><<<ib, 64, 0, st>>>(nbp, h, e.d_hrow, c.bstart, c.blen, c.members,
                                                      c.blk_of, c.loc, c.off, e.d_rowptr, e.d_col, e.d_valf,
                                                      e.d_gdiag, dvec, c.binv, c.flag);
    else
        block_invert_kernel<double><<<ib, 64, 0, st>>>(nbp, h, e.d_hrow, c.bstart, c.blen, c.members,
                                                       c.blk_of, c.loc, c.off, e.d_rowptr, e.d_col, e.d_val,
                                                       e.d_gdiag, dvec, c.binv, c.flag);
    e.launches += 4;
    return check ? precond_check(e, c) : 0;
}

// Waits for the build and checks it: a block count in 1..n and no singular
// block.
int precond_check(Engine &e, const Cluster &c)
{
    int flag = 0, nb = 0;
    cudaMemcpyAsync(&flag, c.flag, sizeof(int), cudaMemcpyDeviceToHost, e.st);
    cudaMemcpyAsync(&nb, c.bbase + e.n, sizeof(int), cudaMemcpyDeviceToHost, e.st);
    if (int rc = e.sync_check("precond build")) return rc;
    if (nb <= 0 || nb > e.n) {
        e.err = "precond: bad block count";
        return SDDDST_ERR_SOLVER;
    }
    if (flag) {
        e.err = "precond: singular cluster block";
        return SDDDST_ERR_SOLVER;
    }
    return 0;
}

void precond_apply(Engine &e, const Cluster &c, const double *v, double *z)
{
    block_apply_kernel<<<(e.n + 255) / 256, 256, 0, e.st>>>(e.n, c.blk_of, c.loc, c.bstart, c.blen, c.members,
                                                            c.off, c.binv, v, z);
    e.launches++;
}

int precond_alloc(Engine &e, Cluster &c)
{
    const int n = e.n;
    int **arrs[] = {&c.ptr, &c.parent, &c.tmp, &c.tmp2, &c.members, &c.blk_of, &c.loc};
    for (int **a : arrs)
        if (cudaMalloc(a, sizeof(int) * n) != cudaSuccess) return SDDDST_ERR_NOMEM;
    int **arrs1[] = {&c.count, &c.fill, &c.start, &c.nblk, &c.bbase, &c.bstart, &c.blen, &c.sq, &c.off};
    for (int **a : arrs1)
        if (cudaMalloc(a, sizeof(int) * (n + 1)) != cudaSuccess) return SDDDST_ERR_NOMEM;
    if (cudaMalloc(&c.flag, sizeof(int)) != cudaSuccess) return SDDDST_ERR_NOMEM;
    return 0;
}

void precond_free(Cluster &c)
{
    int *arrs[] = {c.ptr, c.parent, c.tmp, c.tmp2, c.members, c.blk_of, c.loc, c.count, c.fill, c.start,
                   c.nblk, c.bbase, c.bstart, c.blen, c.sq, c.off, c.flag};
    for (int *a : arrs)
        if (a) cudaFree(a);
    if (c.binv) cudaFree(c.binv);
    c = Cluster{};
}

} // namespace sd
