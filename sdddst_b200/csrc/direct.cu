// Device sparse direct solve of J(h) x = rhs, the drop-in for the UMFPACK
// factorization and solve of Simulation::calculateSparseFormForJacobian /
// solveEQSys (simulation.cpp:386-396): a multifrontal LU over a geometric
// nested dissection of the periodic unit cell.
//
// Ordering.  Two dislocations are coupled in J only when their periodic
// distance is below the pattern radius r_p = (1 + sqrt(36.8)) c
// (simulation.cpp:255-262), so a strip of width w > r_p separates the
// dislocations on its two sides.  The tree splits the torus along x with two
// strips (|x| < w/2 and |x| >= 1/2 - w/2), each half along y the same way,
// then every rectangle across its longer side with one middle strip, down to
// leaves with a side below 3w.  Strips and leaves are the fronts; their
// dislocations are numbered in postorder (children before parents), in
// ascending index inside a front.
//
// Symbolic structure.  What a subtree leaves behind in the Schur complement
// couples ancestor-strip dislocations within r_p of the subtree's rectangle
// (no coupling reaches farther), so each front holds its own dislocations
// plus the ancestor-strip dislocations within w of its rectangle: a superset
// of the exact structure, found by a distance test, exact zeros included.
// A child's set lies inside its parent's front because the child's rectangle
// lies inside the parent's.
//
// Numeric.  Each front is a dense FP64 row-major matrix assembled from the
// rows and columns of J of its own dislocations plus its children's Schur
// complements (extend-add, one child after the other), then partially
// factored in blocks of 64 pivots: row pivoting inside the block, static
// perturbation of pivots below sqrt(eps) of the block's largest entry, the
// triangular inverses of each diagonal block kept for the solves, and an FP64
// tiled update of the trailing matrix.  All fronts at one tree depth share the
// launches.  Row swaps of a block are not applied to the columns left of it:
// the forward solve applies each block's permutation when it reaches the
// block.
//
// Solve.  The forward substitution, leaves to root, passes each front's update
// part to its parent; the backward substitution, root to leaves, reads the
// ancestors' solutions.  The caller refines against the unfactored J
// (residual in FP64, refinement steps, GMRES preconditioned by the factors as
// the last resort).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace sd {

namespace {

constexpr int kNB = 64;          // pivot block
constexpr int kMaxTree = 8191;   // tree nodes
constexpr int kChunk = 256;      // dislocations per ranking chunk
constexpr int kLeafMin = 96;     // expected dislocations below which a rectangle is not split

struct TreeNode {
    int axis;   // split axis (0: x, 1: y), -1: leaf
    int torus;  // split of a periodic axis by two strips
    double lo, hi, cut; // strip [lo, hi); torus: second strip |c| >= cut
    double rx0, rx1, ry0, ry1; // rectangle of the subtree
    int fullx, fully;          // the rectangle spans the period on that axis
    int parent, child0, child1, depth;
};

struct FrontInfo {
    long foff; // front matrix offset (doubles) in the pool
    long ioff; // block inverses offset (doubles)
    long woff; // solve vector offset (doubles)
    int p, u, n, ld;
    int start; // first elimination position of its own dislocations
    int uoff;  // offset of its update list
    int parent, child0, child1, depth;
};

struct Direct {
    // tree (depends on the cutoff only)
    double w = 0.0, built_for = -1.0;
    int T = 0, maxdepth = 0;
    std::vector<TreeNode> tree;
    std::vector<int> postorder;
    TreeNode *d_tree = nullptr;
    // analysis of one Jacobian pattern
    int nchunk = 0;
    int *d_tn = nullptr, *d_lrank = nullptr, *d_ctab = nullptr, *d_cnt = nullptr, *d_pos = nullptr;
    int *d_own = nullptr, *d_perm = nullptr, *d_ucnt = nullptr;
    double *d_xw = nullptr, *d_yw = nullptr, *d_Y = nullptr;
    int *d_upd = nullptr, *d_updpos = nullptr, *d_map = nullptr;
    long upd_cap = 0, updpos_cap = 0, map_cap = 0;
    std::vector<FrontInfo> fr;
    FrontInfo *d_fr = nullptr;
    std::vector<std::vector<int>> levels;
    std::vector<int> level_off, level_pmax, level_nmax, level_umax;
    int *d_levels = nullptr;
    // numeric
    double *d_F = nullptr, *d_inv = nullptr, *d_W = nullptr;
    float *d_Ff = nullptr; // FP32 fronts (SDDDST_SOLVER_DIRECT_MIXED)
    long F_cap = 0, Ff_cap = 0, inv_cap = 0, W_cap = 0, F_used = 0;
    bool f32 = false;
    int *d_npert = nullptr;
    bool analysed = false, factored = false;
    double flops = 0.0; // LU flops of one factorization
    long factorizations = 0, perturbed = 0;
    int *h_buf = nullptr; // pinned
    int h_buf_cap = 0;
    // lookahead: the pivot blocks of outer block J+1 are factored on a
    // high-priority side stream while the main stream updates the rest of
    // the trailing matrix of outer block J
    cudaStream_t side = nullptr;
    cudaEvent_t ev_side = nullptr, ev_next = nullptr, ev_level = nullptr;
};

Direct *D(Engine &e) { return static_cast<Direct *>(e.direct); }

template <typename T> int grow(T *&p, long &cap, long need)
{
    if (need <= cap && p) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    long c = std::max(need, 1L);
    c += c / 8;
    if (cudaMalloc(&p, sizeof(T) * (size_t)c) != cudaSuccess) {
        cap = 0;
        return SDDDST_ERR_NOMEM;
    }
    cap = c;
    return 0;
}

// ------------------------------------------------------------ device helpers

__device__ __forceinline__ double wrap_unit(double v) { return v - rint(v); }

__device__ int tree_assign(const TreeNode *__restrict__ T, double x, double y)
{
    int t = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const TreeNode nd = T[t];
        if (nd.axis < 0) return t;
        const double c = nd.axis == 0 ? x : y;
        if (c >= nd.lo && c < nd.hi) return t;
        if (nd.torus) {
            if (c >= nd.cut || c < -nd.cut) return t;
            t = c < 0.0 ? nd.child0 : nd.child1;
        } else {
            t = c < nd.lo ? nd.child0 : nd.child1;
        }
    }
    return t;
}

__device__ __forceinline__ double axis_gap(double c, double lo, double hi, int full)
{
    if (full || (c >= lo && c < hi)) return 0.0;
    return fmin(fabs(wrap_unit(c - lo)), fabs(wrap_unit(c - hi)));
}

__device__ __forceinline__ bool near_rect(const TreeNode &t, double x, double y, double w)
{
    const double gx = axis_gap(x, t.rx0, t.rx1, t.fullx);
    const double gy = axis_gap(y, t.ry0, t.ry1, t.fully);
    return gx * gx + gy * gy < w * w;
}

// exclusive block scan of one int per thread (blockDim.x == 256)
__device__ int block_scan_excl(int v, int *total)
{
    __shared__ int ws[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __syncthreads();
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k < wid) off += ws[k];
        tot += ws[k];
    }
    *total = tot;
    return off + incl - v;
}

// ------------------------------------------------------------ symbolic kernels

__global__ void assign_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                              const TreeNode *__restrict__ T, int *__restrict__ tn, double *__restrict__ xw,
                              double *__restrict__ yw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = wrap_unit(x[i]), b = wrap_unit(y[i]);
    if (a >= 0.5) a -= 1.0;
    if (b >= 0.5) b -= 1.0;
    xw[i] = a;
    yw[i] = b;
    tn[i] = tree_assign(T, a, b);
}

// rank of each dislocation among the earlier ones of its chunk in the same
// tree node; the last of a node in the chunk writes the chunk's count
__global__ void chunk_rank_kernel(int n, int T, const int *__restrict__ tn, int *__restrict__ lrank,
                                  int *__restrict__ ctab)
{
    __shared__ int s[kChunk];
    const int i = blockIdx.x * kChunk + threadIdx.x;
    s[threadIdx.x] = i < n ? tn[i] : -1;
    __syncthreads();
    if (i >= n) return;
    const int me = s[threadIdx.x];
    int before = 0, after = 0;
    for (int k = 0; k < kChunk; ++k) {
        const int eq = s[k] == me;
        before += (k < (int)threadIdx.x) & eq;
        after += (k > (int)threadIdx.x) & eq;
    }
    lrank[i] = before;
    if (after == 0) ctab[(long)blockIdx.x * T + me] = before + 1;
}

__global__ void chunk_scan_kernel(int T, int nchunk, int *__restrict__ ctab, int *__restrict__ cnt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    int run = 0;
    for (int c = 0; c < nchunk; ++c) {
        const int v = ctab[(long)c * T + t];
        ctab[(long)c * T + t] = run;
        run += v;
    }
    cnt[t] = run;
}

__global__ void place_kernel(int n, int T, const int *__restrict__ tn, const int *__restrict__ lrank,
                             const int *__restrict__ ctab, const FrontInfo *__restrict__ fr, int *__restrict__ pos,
                             int *__restrict__ own)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = tn[i];
    const int q = fr[t].start + ctab[(long)(i / kChunk) * T + t] + lrank[i];
    pos[i] = q;
    own[q] = i;
}

// update sets: ancestor-strip dislocations within w of the node's rectangle,
// nearest ancestor first (ascending elimination position)
template <bool kFill>
__global__ void update_set_kernel(const TreeNode *__restrict__ T, const FrontInfo *__restrict__ fr,
                                  const int *__restrict__ own, const double *__restrict__ xw,
                                  const double *__restrict__ yw, double w, int *__restrict__ ucnt,
                                  int *__restrict__ upd, int *__restrict__ updpos)
{
    const int t = blockIdx.x;
    const TreeNode me = T[t];
    int count = 0;
    int base = kFill ? fr[t].uoff : 0;
    for (int a = me.parent; a >= 0; a = T[a].parent) {
        const int s0 = fr[a].start, pa = fr[a].p;
        for (int k0 = 0; k0 < pa; k0 += 256) {
            const int k = k0 + threadIdx.x;
            int j = -1, hit = 0;
            if (k < pa) {
                j = own[s0 + k];
                hit = near_rect(me, xw[j], yw[j], w) ? 1 : 0;
            }
            int tot;
            const int off = block_scan_excl(hit, &tot);
            if (kFill && hit) {
                upd[base + count + off] = j;
                updpos[base + count + off] = s0 + k;
            }
            count += tot;
        }
    }
    if (!kFill && threadIdx.x == 0) ucnt[t] = count;
}

__device__ __forceinline__ int find_sorted(const int *__restrict__ a, int len, int key)
{
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return (lo < len && a[lo] == key) ? lo : -1;
}

// local index of elimination position q in front f (-1: not in the front)
__device__ __forceinline__ int front_local(const FrontInfo &f, const int *__restrict__ updpos, int q)
{
    if (q >= f.start && q < f.start + f.p) return q - f.start;
    const int k = find_sorted(updpos + f.uoff, f.u, q);
    return k < 0 ? -1 : f.p + k;
}

__global__ void map_kernel(int T, const FrontInfo *__restrict__ fr, const int *__restrict__ updpos,
                           int *__restrict__ map, int *__restrict__ flag)
{
    const int c = blockIdx.x;
    const FrontInfo fc = fr[c];
    if (fc.parent < 0) return;
    const FrontInfo fp = fr[fc.parent];
    for (int q = threadIdx.x; q < fc.u; q += blockDim.x) {
        int l = front_local(fp, updpos, updpos[fc.uoff + q]);
        if (l < 0) {
            atomicExch(flag, 2);
            l = 0;
        }
        map[fc.uoff + q] = l;
    }
}

// ------------------------------------------------------------ numeric kernels

// rows and columns of J of each front's own dislocations; one warp per row
template <typename VT, typename FT>
__global__ void assemble_kernel(int n, double h, const int *__restrict__ rowptr, const int *__restrict__ col,
                                const VT *__restrict__ val, const double *__restrict__ gdiag,
                                const double *__restrict__ dvec, const int *__restrict__ tn,
                                const int *__restrict__ pos, const FrontInfo *__restrict__ fr,
                                const int *__restrict__ updpos, FT *__restrict__ F, int *__restrict__ flag)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const FrontInfo f = fr[tn[i]];
    FT *Ff = F + f.foff;
    const int li = pos[i] - f.start;
    const double di = (1.0 + dvec[i]) * 0.5 * h;
    const int s = rowptr[i], e = rowptr[i + 1];
    for (int q = s + lane; q < e; q += 32) {
        const int j = col[q];
        if (j == i) {
            Ff[(long)li * f.ld + li] = (FT)(1.0 + di * gdiag[i]);
            continue;
        }
        const int pj = pos[j];
        if (pj < f.start) continue; // a descendant: assembled in its own front
        const int lj = front_local(f, updpos, pj);
        if (lj < 0) {
            atomicExch(flag, 3);
            continue;
        }
        const double g = (double)val[q];
        Ff[(long)li * f.ld + lj] = (FT)(di * g);
        if (lj >= f.p) Ff[(long)lj * f.ld + li] = (FT)((1.0 + dvec[j]) * 0.5 * h * g);
    }
}

// parent += child's Schur complement, for the child in one slot
template <typename FT>
__global__ void extend_add_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list, int slot,
                                  FT *__restrict__ F, const int *__restrict__ map)
{
    const FrontInfo ft = fr[list[blockIdx.y]];
    const int c = slot ? ft.child1 : ft.child0;
    if (c < 0) return;
    const FrontInfo fc = fr[c];
    const int tiles = (fc.u + 31) >> 5;
    if ((int)blockIdx.x >= tiles * tiles) return;
    const int a0 = (blockIdx.x / tiles) * 32, b0 = (blockIdx.x % tiles) * 32;
    __shared__ int mr[32], mc[32];
    if (threadIdx.x < 32) mr[threadIdx.x] = a0 + threadIdx.x < fc.u ? map[fc.uoff + a0 + threadIdx.x] : 0;
    else if (threadIdx.x < 64) {
        const int k = threadIdx.x - 32;
        mc[k] = b0 + k < fc.u ? map[fc.uoff + b0 + k] : 0;
    }
    __syncthreads();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const FT *Fc = F + fc.foff;
    FT *Ft = F + ft.foff;
    for (int r = ty; r < 32; r += 8) {
        const int a = a0 + r, b = b0 + tx;
        if (a < fc.u && b < fc.u)
            Ft[(long)mr[r] * ft.ld + mc[tx]] += Fc[(long)(fc.p + a) * fc.ld + fc.p + b];
    }
}

// LU of the diagonal block of pivot block j (row pivoting inside the block),
// its triangular inverses, and the block-local row permutation
constexpr int kDiagThreads = 256;

template <typename FT>
__global__ void __launch_bounds__(kDiagThreads) diag_block_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list,
                                                         int j, FT *__restrict__ F, double *__restrict__ inv,
                                                         int *__restrict__ perm, int *__restrict__ npert)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = j * kNB;
    if (s >= f.p) return;
    const int b = min(kNB, f.p - s);
    extern __shared__ double sm[];
    double(*Dm)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double(*Li)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + kNB * (kNB + 1));
    double(*Ui)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + 2 * kNB * (kNB + 1));
    __shared__ int pv[kNB];
    __shared__ int piv;
    __shared__ double red[8];
    FT *Ff = F + f.foff;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double amax = 0.0;
    for (int idx = tid; idx < kNB * kNB; idx += 256) {
        const int r = idx >> 6, c = idx & 63;
        const double v = (r < b && c < b) ? (double)Ff[(long)(s + r) * f.ld + s + c] : 0.0;
        Dm[r][c] = v;
        amax = fmax(amax, fabs(v));
    }
    if (tid < kNB) pv[tid] = tid;
    amax = warp_max(amax);
    if (lane == 0) red[wid] = amax;
    __syncthreads();
    amax = red[0];
    for (int k = 1; k < 8; ++k) amax = fmax(amax, red[k]);
    const double thr = 1.4901161193847656e-08 * (amax > 0.0 ? amax : 1.0);
    int pert = 0;
    for (int c = 0; c < b; ++c) {
        if (wid == 0) {
            double best = -1.0;
            int br = c;
            for (int r = c + lane; r < b; r += 32) {
                const double v = fabs(Dm[r][c]);
                if (v > best) {
                    best = v;
                    br = r;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int orr = __shfl_xor_sync(0xffffffffu, br, o);
                if (ob > best || (ob == best && orr < br)) {
                    best = ob;
                    br = orr;
                }
            }
            if (lane == 0) piv = br;
        }
        __syncthreads();
        const int pr = piv;
        if (pr != c) {
            if (tid < b) {
                const double t = Dm[c][tid];
                Dm[c][tid] = Dm[pr][tid];
                Dm[pr][tid] = t;
            }
            if (tid == 0) {
                const int t = pv[c];
                pv[c] = pv[pr];
                pv[pr] = t;
            }
        }
        __syncthreads();
        double d = Dm[c][c];
        if (!(fabs(d) >= thr)) {
            d = d < 0.0 ? -thr : thr;
            pert = 1;
        }
        __syncthreads();
        if (tid == 0) Dm[c][c] = d;
        for (int r = c + 1 + tid; r < b; r += 256) Dm[r][c] /= d;
        __syncthreads();
        // rank-1 update on a 16 x 16 thread grid (no index division)
        for (int r = c + 1 + (tid >> 4); r < b; r += 16) {
            const double l = Dm[r][c];
            for (int cc = c + 1 + (tid & 15); cc < b; cc += 16) Dm[r][cc] = fma(-l, Dm[c][cc], Dm[r][cc]);
        }
        __syncthreads();
        if (tid == 0 && pert) {
            atomicAdd(npert, 1);
            pert = 0;
        }
    }
    // inverses: thread c < 64 owns column c of L^-1, thread 64 + c column c of U^-1
    if (tid < kNB) {
        const int c = tid;
        for (int r = 0; r < kNB; ++r) Li[r][c] = r == c ? 1.0 : 0.0;
        if (c < b)
            for (int r = c + 1; r < b; ++r) {
                double acc = Dm[r][c];
                for (int k = c + 1; k < r; ++k) acc = fma(Dm[r][k], Li[k][c], acc);
                Li[r][c] = -acc;
            }
    } else if (tid < 2 * kNB) {
        const int c = tid - kNB;
        for (int r = 0; r < kNB; ++r) Ui[r][c] = 0.0;
        if (c < b) {
            Ui[c][c] = 1.0 / Dm[c][c];
            for (int r = c - 1; r >= 0; --r) {
                double acc = 0.0;
                for (int k = r + 1; k <= c; ++k) acc = fma(Dm[r][k], Ui[k][c], acc);
                Ui[r][c] = -acc / Dm[r][r];
            }
        }
    }
    __syncthreads();
    for (int idx = tid; idx < kNB * kNB; idx += 256) {
        const int r = idx >> 6, c = idx & 63;
        if (r < b && c < b) Ff[(long)(s + r) * f.ld + s + c] = (FT)Dm[r][c];
    }
    double *L = inv + f.ioff + (long)j * 2 * kNB * kNB;
    double *U = L + kNB * kNB;
    for (int idx = tid; idx < kNB * kNB; idx += 256) {
        const int r = idx / kNB, c = idx % kNB;
        L[idx] = Li[r][c];
        U[idx] = Ui[r][c];
    }
    if (tid < b) perm[f.start + s + tid] = pv[tid];
}

// Pivot block j's row panel U12 = L11^-1 P A12 over a column range (the first
// `uhalf` CTAs of the grid, 64 columns each) and its column panel
// L21 = A21 U11^-1 for rows e..n (the other CTAs, when `lrows` is set).
// Column ranges of the U12 part: umode 1: [e, e1), up to the end of the
// 128-pivot outer block; umode 2: [e1, n), deferred until the outer block's
// second pivot block is factored; umode 3: [e, n).
template <typename FT>
__global__ void __launch_bounds__(256) panel_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list,
                                                    int j, FT *__restrict__ F, const double *__restrict__ inv,
                                                    const int *__restrict__ perm, int umode, int uhalf, int lrows)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = j * kNB;
    if (s >= f.p) return;
    const int b = min(kNB, f.p - s), e = s + b;
    const int e1 = min(f.p, (j >> 1) * 2 * kNB + 2 * kNB);
    const bool upper = (int)blockIdx.x < uhalf;
    int lo, hi;
    if (upper) {
        lo = umode == 2 ? e1 : e;
        hi = umode == 1 ? e1 : f.n;
    } else {
        if (!lrows) return;
        lo = e;
        hi = f.n;
    }
    const int tile = upper ? blockIdx.x : blockIdx.x - uhalf;
    const int t0 = tile * kNB;
    if (lo + t0 >= hi) return;
    const int cnt = min(kNB, hi - lo - t0);
    extern __shared__ double sm[];
    double(*Xs)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double(*As)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + kNB * (kNB + 1));
    FT *Ff = F + f.foff;
    const double *Lb = inv + f.ioff + (long)j * 2 * kNB * kNB;
    const double *Xg = upper ? Lb : Lb + kNB * kNB;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kNB * kNB; idx += 256) Xs[idx / kNB][idx % kNB] = Xg[idx];
    if (upper) {
        for (int idx = tid; idx < kNB * kNB; idx += 256) {
            const int k = idx / kNB, c = idx % kNB;
            As[k][c] = (k < b && c < cnt) ? (double)Ff[(long)(s + perm[f.start + s + k]) * f.ld + lo + t0 + c] : 0.0;
        }
    } else {
        for (int idx = tid; idx < kNB * kNB; idx += 256) {
            const int r = idx / kNB, k = idx % kNB;
            As[r][k] = (r < cnt && k < b) ? (double)Ff[(long)(lo + t0 + r) * f.ld + s + k] : 0.0;
        }
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
    if (upper) {
        // R[i][c] = sum_k Linv[i][k] A[k][c]
        for (int k = 0; k < b; ++k) {
            double xv[4], av[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xv[a] = Xs[ty * 4 + a][k];
#pragma unroll
            for (int c = 0; c < 4; ++c) av[c] = As[k][tx + 16 * c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] = fma(xv[a], av[c], acc[a][c]);
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int i = ty * 4 + a, cc = tx + 16 * c;
                if (i < b && cc < cnt) Ff[(long)(s + i) * f.ld + lo + t0 + cc] = (FT)acc[a][c];
            }
    } else {
        // R[r][jj] = sum_k A[r][k] Uinv[k][jj]
        for (int k = 0; k < b; ++k) {
            double av[4], xv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = As[ty * 4 + a][k];
#pragma unroll
            for (int c = 0; c < 4; ++c) xv[c] = Xs[k][tx + 16 * c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] = fma(av[a], xv[c], acc[a][c]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int r = ty * 4 + a, jj = tx + 16 * c;
                if (r < cnt && jj < b) Ff[(long)(lo + t0 + r) * f.ld + s + jj] = (FT)acc[a][c];
            }
    }
}

// Updates of the trailing matrix by outer block J (pivot blocks 2J and 2J+1,
// columns [s0, e0) and [e0, e1)):
//   mode 0: rows [e0, n) x columns [e0, e1), K = [s0, e0)  (second pivot block's columns);
//   mode 1: rows [e0, e1) x columns [e1, n), K = [s0, e0)  (second pivot block's rows);
//   mode 2: rows [e1, n) x columns [e1, s0 + 256), K = [s0, e1)  (the next outer block's columns);
//   mode 3: rows [e1, n) x columns [s0 + 256, n), K = [s0, e1)  (the rest of the trailing matrix).
// 128 x 128 tiles, 8 x 8 outputs per thread; K in chunks of 16 double-buffered
// in shared memory by cp.async (element-sized copies, zero-filled outside the
// ranges); the accumulators start from C (independent loads in flight with
// the first copy), so C is read and written once per outer block.  FP64
// fronts: one CTA per SM (8 x 8 FP64 accumulators); FP32 fronts: two.
constexpr int kBM = 128, kBK = 16;
template <typename FT> __host__ __device__ constexpr int upd_pad() { return 16 / (int)sizeof(FT); } // keeps rows 16-byte aligned
template <typename FT> constexpr size_t upd_smem() { return 4 * kBK * (kBM + upd_pad<FT>()) * sizeof(FT); }

template <typename FT> __device__ __forceinline__ void cp_async_el(void *smem, const void *gmem, bool pred)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = pred ? (int)sizeof(FT) : 0;
    if (sizeof(FT) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ld4(const double *p, double v[4])
{
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, float v[4])
{
    const float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

template <typename FT>
__global__ void __launch_bounds__(256, sizeof(FT) == 4 ? 2 : 1)
    update_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list, int J, int mode, FT *__restrict__ F)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = J * 2 * kNB;
    if (s >= f.p) return;
    const int e0 = s + min(kNB, f.p - s), e1 = min(f.p, s + 2 * kNB);
    int rlo, rhi, clo, chi, kend;
    if (mode == 0) {
        rlo = e0; rhi = f.n; clo = e0; chi = e1; kend = e0;
    } else if (mode == 1) {
        rlo = e0; rhi = e1; clo = e1; chi = f.n; kend = e0;
    } else if (mode == 2) {
        rlo = e1; rhi = f.n; clo = e1; chi = min(f.n, s + 4 * kNB); kend = e1;
    } else {
        rlo = e1; rhi = f.n; clo = s + 4 * kNB; chi = f.n; kend = e1;
    }
    if (rlo >= rhi || clo >= chi) return;
    const int b = kend - s;
    const int tm = (rhi - rlo + kBM - 1) / kBM, tn = (chi - clo + kBM - 1) / kBM;
    if ((int)blockIdx.x >= tm * tn) return;
    const int row0 = rlo + (blockIdx.x / tn) * kBM, col0 = clo + (blockIdx.x % tn) * kBM;
    constexpr int kP = upd_pad<FT>();
    typedef FT Tile[kBK][kBM + kP];
    extern __shared__ __align__(16) unsigned char smraw[];
    Tile *As = reinterpret_cast<Tile *>(smraw);
    Tile *Bs = reinterpret_cast<Tile *>(smraw + 2 * sizeof(Tile));
    FT *Ff = F + f.foff;
    const long ld = f.ld;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    // thread tid copies A rows (tid >> 4) + 16 q, column tid & 15, and B rows
    // (tid >> 7) + 2 q, column tid & 127, of each chunk (q = 0..7)
    const int ar = tid >> 4, ak = tid & 15, bk = tid >> 7, bc = tid & 127;
    const FT *gA = Ff + (long)(row0 + ar) * ld + s + ak;
    const FT *gB = Ff + (long)(s + bk) * ld + col0 + bc;
    const bool colB_ok = col0 + bc < chi;
    auto issue = [&](int buf, int k0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const bool pa = row0 + ar + 16 * q < rhi && k0 + ak < b;
            cp_async_el<FT>(&As[buf][ak][ar + 16 * q], pa ? gA + (long)16 * q * ld + k0 : Ff, pa);
            const bool pb = k0 + bk + 2 * q < b && colB_ok;
            cp_async_el<FT>(&Bs[buf][bk + 2 * q][bc], pb ? gB + (long)(k0 + 2 * q) * ld : Ff, pb);
        }
        cp_async_commit();
    };
    const int nk = (b + kBK - 1) / kBK;
    issue(0, 0);
    FT acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int r = row0 + (a < 4 ? ty * 4 + a : 64 + ty * 4 + a - 4);
        const FT *row = Ff + (long)min(r, rhi - 1) * ld;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cc = col0 + (c < 4 ? tx * 4 + c : 64 + tx * 4 + c - 4);
            acc[a][c] = (r < rhi && cc < chi) ? row[cc] : (FT)0;
        }
    }
    for (int kc = 0; kc < nk; ++kc) {
        if (kc + 1 < nk) {
            issue((kc + 1) & 1, (kc + 1) * kBK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const Tile &A = As[kc & 1];
        const Tile &B = Bs[kc & 1];
#pragma unroll
        for (int k = 0; k < kBK; ++k) {
            FT av[8], bv[8];
            ld4(&A[k][ty * 4], av);
            ld4(&A[k][64 + ty * 4], av + 4);
            ld4(&B[k][tx * 4], bv);
            ld4(&B[k][64 + tx * 4], bv + 4);
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[a][c] = fma(-av[a], bv[c], acc[a][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int r = row0 + (a < 4 ? ty * 4 + a : 64 + ty * 4 + a - 4);
        if (r >= rhi) continue;
        FT *row = Ff + (long)r * ld;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cc = col0 + (c < 4 ? tx * 4 + c : 64 + tx * 4 + c - 4);
            if (cc < chi) row[cc] = acc[a][c];
        }
    }
}

// The same trailing update for FP32 fronts on the 5th-gen tensor cores
// (tcgen05, kind::tf32): one CTA of 128 threads per 128 x 128 tile of C,
// D = A B accumulated in FP32 in tensor memory, C -= D in the epilogue.  A
// TF32 operand keeps 10 mantissa bits, so the product is compensated: with
// A_lo = A - tf32(A) and B_lo = B - tf32(B) (exact in FP32),
//   A B ~ A B + A B_lo + A_lo B   (tf32 parts; the dropped A_lo B_lo is
// below 2^-20 of A B), which keeps the factors near FP32 accuracy and the
// FP64 refinement at its usual step count.  K runs in chunks of 32: A, A_lo
// (128 x 32) and B, B_lo (transposed to 128 x 32) are staged in shared memory
// in the no-swizzle K-major core-matrix layout (8 rows x 16 bytes per core
// matrix, K-adjacent ones 128 bytes apart, 8-row groups 1024 bytes apart);
// a warp covers 8 rows x 4 K per store, so its 32 lanes write 128
// contiguous bytes.  The next chunk's global loads are issued into registers
// before the CTA waits for the current chunk's MMAs (one thread issues 3 x 4
// MMAs, M = N = 128, K = 8, and commits them to an mbarrier; bounded wait,
// past the limit *err is set and the tile is left unchanged).  The epilogue
// moves D through shared memory (rows padded to 129 words) so that C is read
// and written row-contiguously.  Same modes and tile order as update_kernel.
constexpr int kTcK = 32;                                  // K chunk
constexpr unsigned kTcOp = 128 * kTcK * 4;                // one staged operand: 16 KB
constexpr size_t kTcSmem = 68 * 1024;                     // A, A_lo, B, B_lo or D (128 x 129 words), aligned

__device__ __forceinline__ unsigned long long tc_desc(unsigned addr)
{
    // start address, leading byte offset 128 (K-adjacent core matrices),
    // stride byte offset 1024 (8-row groups), version 1, no swizzle
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)(128u >> 4) << 16) |
           ((unsigned long long)(1024u >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ float tf32_lo(float v) // v - (v with its low 13 mantissa bits cleared)
{
    return v - __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
}

__global__ void __launch_bounds__(128)
    update_tc_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list, int J, int mode,
                     float *__restrict__ F, int *__restrict__ err)
{
    // instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, N = 128, M = 128
    constexpr unsigned kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = J * 2 * kNB;
    if (s >= f.p) return;
    const int e0 = s + min(kNB, f.p - s), e1 = min(f.p, s + 2 * kNB);
    int rlo, rhi, clo, chi, kend;
    if (mode == 0) {
        rlo = e0; rhi = f.n; clo = e0; chi = e1; kend = e0;
    } else if (mode == 1) {
        rlo = e0; rhi = e1; clo = e1; chi = f.n; kend = e0;
    } else if (mode == 2) {
        rlo = e1; rhi = f.n; clo = e1; chi = min(f.n, s + 4 * kNB); kend = e1;
    } else {
        rlo = e1; rhi = f.n; clo = s + 4 * kNB; chi = f.n; kend = e1;
    }
    if (rlo >= rhi || clo >= chi) return;
    const int b = kend - s;
    const int tm = (rhi - rlo + kBM - 1) / kBM, tn = (chi - clo + kBM - 1) / kBM;
    if ((int)blockIdx.x >= tm * tn) return; // whole CTA: before any barrier or allocation
    const int row0 = rlo + (blockIdx.x / tn) * kBM, col0 = clo + (blockIdx.x % tn) * kBM;
    extern __shared__ __align__(16) unsigned char tcs_raw[];
    unsigned char *tcs = tcs_raw + ((1024u - ((unsigned)__cvta_generic_to_shared(tcs_raw) & 1023u)) & 1023u);
    unsigned char *sA = tcs, *sAl = tcs + kTcOp, *sB = tcs + 2 * kTcOp, *sBl = tcs + 3 * kTcOp;
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float *Ff = F + f.foff;
    const long ld = f.ld;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (unsigned)__cvta_generic_to_shared(&tmem_slot)),
                     "r"(128u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(&mbar)),
                     "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_slot;
    const unsigned mb = (unsigned)__cvta_generic_to_shared(&mbar);
    const int nk = (b + kTcK - 1) / kTcK;
    // step `it` of a warp covers 8 rows (lane >> 2) x 4 K (lane & 3) of core
    // matrix group g = 4 it + warp: row group g >> 3, K quad g & 7
    const int lr = lane >> 2, lk = lane & 3;
    float ra[32], rb[32];
    auto load_chunk = [&](int k0) {
#pragma unroll
        for (int it = 0; it < 32; ++it) {
            const int g = 4 * it + warp, r8 = g >> 3, kq = g & 7;
            const int r = r8 * 8 + lr, k = k0 + kq * 4 + lk;
            ra[it] = (k < b && row0 + r < rhi) ? Ff[(long)(row0 + r) * ld + s + k] : 0.0f;
            rb[it] = (k < b && col0 + r < chi) ? Ff[(long)(s + k) * ld + col0 + r] : 0.0f;
        }
    };
    load_chunk(0);
    bool ok = true;
    for (int kc = 0; kc < nk && ok; ++kc) {
#pragma unroll
        for (int it = 0; it < 32; ++it) {
            const int g = 4 * it + warp;
            const unsigned o = (unsigned)((g >> 3) * 1024 + (g & 7) * 128 + lane * 4);
            *reinterpret_cast<float *>(sA + o) = ra[it];
            *reinterpret_cast<float *>(sAl + o) = tf32_lo(ra[it]);
            *reinterpret_cast<float *>(sB + o) = rb[it];
            *reinterpret_cast<float *>(sBl + o) = tf32_lo(rb[it]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const unsigned a0 = (unsigned)__cvta_generic_to_shared(sA), al0 = (unsigned)__cvta_generic_to_shared(sAl);
            const unsigned b0 = (unsigned)__cvta_generic_to_shared(sB), bl0 = (unsigned)__cvta_generic_to_shared(sBl);
#pragma unroll
            for (int t = 0; t < kTcK / 8; ++t) {
                const unsigned off = 256u * t;
                const unsigned long long pa[3] = {tc_desc(a0 + off), tc_desc(a0 + off), tc_desc(al0 + off)};
                const unsigned long long pb[3] = {tc_desc(b0 + off), tc_desc(bl0 + off), tc_desc(b0 + off)};
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const unsigned acc = (kc > 0 || t > 0 || q > 0) ? 1u : 0u;
                    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                                 "l"(pa[q]), "l"(pb[q]), "r"(kIdesc), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        // the next chunk's loads in flight while the MMAs run
        if (kc + 1 < nk) load_chunk((kc + 1) * kTcK);
        unsigned done = 0;
        for (int it = 0; it < (1 << 22) && !done; ++it) {
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}"
                         : "=r"(done)
                         : "r"(mb), "r"((unsigned)(kc & 1))
                         : "memory");
            if (!done && it > 32) __nanosleep(64);
        }
        ok = __syncthreads_and(done) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // D through shared memory (the operands are no longer read): warp w
        // holds rows 32 w .. 32 w + 31 of D, one TMEM lane each
        float *Ds = reinterpret_cast<float *>(tcs);
        const int r = warp * 32 + lane;
        const unsigned lane_base = (unsigned)(warp * 32) << 16;
#pragma unroll 1
        for (int c0 = 0; c0 < kBM; c0 += 16) {
            unsigned v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + lane_base + (unsigned)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) Ds[r * 129 + c0 + q] = __uint_as_float(v[q]);
        }
        __syncthreads();
        // C -= D, a warp per row at a time, columns contiguous
        for (int rr = warp; rr < kBM; rr += 4) {
            const int gr = row0 + rr;
            if (gr >= rhi) break;
            float *row = Ff + (long)gr * ld + col0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int c = lane + 32 * q;
                if (col0 + c < chi) row[c] -= Ds[rr * 129 + c];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
}

// ------------------------------------------------------------ solve kernels

// forward, per front: own part from the right-hand side, update part zero,
// plus the children's passed-up parts (child 0, then child 1)
__global__ void fgather_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list,
                               const int *__restrict__ own, const int *__restrict__ map,
                               const double *__restrict__ rhs, double *__restrict__ W)
{
    const FrontInfo f = fr[list[blockIdx.x]];
    double *w = W + f.woff;
    for (int k = threadIdx.x; k < f.n; k += blockDim.x) w[k] = k < f.p ? rhs[own[f.start + k]] : 0.0;
    __syncthreads();
    for (int slot = 0; slot < 2; ++slot) {
        const int c = slot ? f.child1 : f.child0;
        if (c < 0) continue;
        const FrontInfo fc = fr[c];
        const double *wc = W + fc.woff + fc.p;
        for (int q = threadIdx.x; q < fc.u; q += blockDim.x) w[map[fc.uoff + q]] += wc[q];
        __syncthreads();
    }
}

constexpr int kRowsPerCta = 64;

__device__ __forceinline__ void small_matvec(const double *__restrict__ M, const double *__restrict__ v, double *out,
                                             int b)
{
    // out[i] = sum_k M[i][k] v[k] for i < b (M row-major 64 x 64, zeros outside its triangle)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = wid; i < b; i += 8) {
        double acc = 0.0;
        if (lane < b) acc = M[i * kNB + lane] * v[lane];
        if (lane + 32 < b) acc = fma(M[i * kNB + lane + 32], v[lane + 32], acc);
        acc = warp_sum(acc);
        if (lane == 0) out[i] = acc;
    }
}

template <typename FT>
__global__ void fblock_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list, int j,
                              const FT *__restrict__ F, const double *__restrict__ inv,
                              const int *__restrict__ perm, double *__restrict__ W, double *__restrict__ Y)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = j * kNB;
    if (s >= f.p) return;
    const int b = min(kNB, f.p - s), e = s + b;
    const int r0 = e + blockIdx.x * kRowsPerCta;
    if (blockIdx.x > 0 && r0 >= f.n) return;
    __shared__ double pw[kNB], yb[kNB];
    double *w = W + f.woff;
    if (threadIdx.x < kNB) pw[threadIdx.x] = threadIdx.x < b ? w[s + perm[f.start + s + threadIdx.x]] : 0.0;
    __syncthreads();
    small_matvec(inv + f.ioff + (long)j * 2 * kNB * kNB, pw, yb, b);
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x < b) Y[f.start + s + threadIdx.x] = yb[threadIdx.x];
    const FT *Ff = F + f.foff;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int r = r0 + wid; r < min(f.n, r0 + kRowsPerCta); r += 8) {
        const FT *row = Ff + (long)r * f.ld + s;
        double acc = 0.0;
        if (lane < b) acc = (double)row[lane] * yb[lane];
        if (lane + 32 < b) acc = fma((double)row[lane + 32], yb[lane + 32], acc);
        acc = warp_sum(acc);
        if (lane == 0) w[r] -= acc;
    }
}

// backward, per front: z = y - U12 x_update into the own part of W
template <typename FT>
__global__ void bupdate_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list,
                               const FT *__restrict__ F, const int *__restrict__ upd,
                               const double *__restrict__ Y, const double *__restrict__ X, double *__restrict__ W)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int r0 = blockIdx.x * kRowsPerCta;
    if (r0 >= f.p) return;
    const FT *Ff = F + f.foff;
    double *w = W + f.woff;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int r = r0 + wid; r < min(f.p, r0 + kRowsPerCta); r += 8) {
        const FT *row = Ff + (long)r * f.ld + f.p;
        double acc = 0.0;
        for (int q = lane; q < f.u; q += 32) acc = fma((double)row[q], X[upd[f.uoff + q]], acc);
        acc = warp_sum(acc);
        if (lane == 0) w[r] = Y[f.start + r] - acc;
    }
}

template <typename FT>
__global__ void bblock_kernel(const FrontInfo *__restrict__ fr, const int *__restrict__ list, int j,
                              const FT *__restrict__ F, const double *__restrict__ inv,
                              const int *__restrict__ own, double *__restrict__ W, double *__restrict__ X)
{
    const FrontInfo f = fr[list[blockIdx.y]];
    const int s = j * kNB;
    if (s >= f.p) return;
    const int b = min(kNB, f.p - s);
    const int r0 = blockIdx.x * kRowsPerCta;
    if (blockIdx.x > 0 && r0 >= s) return;
    __shared__ double zb[kNB], xb[kNB];
    double *w = W + f.woff;
    if (threadIdx.x < kNB) zb[threadIdx.x] = threadIdx.x < b ? w[s + threadIdx.x] : 0.0;
    __syncthreads();
    small_matvec(inv + f.ioff + (long)j * 2 * kNB * kNB + kNB * kNB, zb, xb, b);
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x < b) X[own[f.start + s + threadIdx.x]] = xb[threadIdx.x];
    const FT *Ff = F + f.foff;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int r = r0 + wid; r < min(s, r0 + kRowsPerCta); r += 8) {
        const FT *row = Ff + (long)r * f.ld + s;
        double acc = 0.0;
        if (lane < b) acc = (double)row[lane] * xb[lane];
        if (lane + 32 < b) acc = fma((double)row[lane + 32], xb[lane + 32], acc);
        acc = warp_sum(acc);
        if (lane == 0) w[r] -= acc;
    }
}

__global__ void resid_kernel(int n, const double *__restrict__ rhs, const double *__restrict__ jx,
                             double *__restrict__ r)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = rhs[i] - jx[i];
}

__global__ void addto_kernel(int n, const double *__restrict__ z, double *__restrict__ x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += z[i];
}

constexpr size_t kDiagSmem = 3 * kNB * (kNB + 1) * sizeof(double);
constexpr size_t kPanelSmem = 2 * kNB * (kNB + 1) * sizeof(double);

// ------------------------------------------------------------ host: tree

void build_tree(Direct &d, const Engine &e)
{
    const double rp = e.cutoff * (1.0 + std::sqrt(36.8));
    d.w = rp * (1.0 + 1e-6) + 1e-12;
    const double w = d.w;
    d.tree.clear();
    TreeNode root{};
    root.axis = -1;
    root.fullx = root.fully = 1;
    root.rx0 = root.ry0 = -0.5;
    root.rx1 = root.ry1 = 0.5;
    root.parent = root.child0 = root.child1 = -1;
    d.tree.push_back(root);
    std::vector<int> stack{0};
    while (!stack.empty()) {
        const int t = stack.back();
        stack.pop_back();
        TreeNode nd = d.tree[t];
        if ((int)d.tree.size() + 2 > kMaxTree || nd.depth >= 40) continue;
        int axis = -1, torus = 0;
        if (nd.fullx || nd.fully) {
            if (w < 0.4) {
                axis = nd.fullx ? 0 : 1;
                torus = 1;
            }
        } else {
            const double lx = nd.rx1 - nd.rx0, ly = nd.ry1 - nd.ry0;
            const double L = std::max(lx, ly);
            if (L >= 3.0 * w && (double)e.n * lx * ly >= kLeafMin) axis = lx >= ly ? 0 : 1;
        }
        if (axis < 0) continue;
        TreeNode c0 = nd, c1 = nd;
        c0.axis = c1.axis = -1;
        c0.torus = c1.torus = 0;
        c0.parent = c1.parent = t;
        c0.child0 = c0.child1 = c1.child0 = c1.child1 = -1;
        c0.depth = c1.depth = nd.depth + 1;
        nd.axis = axis;
        nd.torus = torus;
        if (torus) {
            nd.lo = -0.5 * w;
            nd.hi = 0.5 * w;
            nd.cut = 0.5 - 0.5 * w;
            if (axis == 0) {
                c0.fullx = c1.fullx = 0;
                c0.rx0 = -nd.cut; c0.rx1 = nd.lo;
                c1.rx0 = nd.hi;   c1.rx1 = nd.cut;
            } else {
                c0.fully = c1.fully = 0;
                c0.ry0 = -nd.cut; c0.ry1 = nd.lo;
                c1.ry0 = nd.hi;   c1.ry1 = nd.cut;
            }
        } else {
            const double a0 = axis == 0 ? nd.rx0 : nd.ry0, a1 = axis == 0 ? nd.rx1 : nd.ry1;
            const double mid = 0.5 * (a0 + a1);
            nd.lo = mid - 0.5 * w;
            nd.hi = mid + 0.5 * w;
            nd.cut = 0.0;
            if (axis == 0) {
                c0.rx1 = nd.lo;
                c1.rx0 = nd.hi;
            } else {
                c0.ry1 = nd.lo;
                c1.ry0 = nd.hi;
            }
        }
        nd.child0 = (int)d.tree.size();
        nd.child1 = nd.child0 + 1;
        d.tree[t] = nd;
        d.tree.push_back(c0);
        d.tree.push_back(c1);
        stack.push_back(nd.child0);
        stack.push_back(nd.child1);
    }
    d.T = (int)d.tree.size();
    // postorder
    d.postorder.clear();
    std::vector<std::pair<int, int>> st{{0, 0}};
    while (!st.empty()) {
        auto &top = st.back();
        const TreeNode &nd = d.tree[top.first];
        if (nd.axis >= 0 && top.second < 2) {
            const int c = top.second == 0 ? nd.child0 : nd.child1;
            top.second++;
            st.push_back({c, 0});
        } else {
            d.postorder.push_back(top.first);
            st.pop_back();
        }
    }
    d.maxdepth = 0;
    for (const auto &nd : d.tree) d.maxdepth = std::max(d.maxdepth, nd.depth);
    d.levels.assign(d.maxdepth + 1, {});
    for (int t = 0; t < d.T; ++t) d.levels[d.tree[t].depth].push_back(t);
    d.level_off.assign(d.maxdepth + 2, 0);
    std::vector<int> flat;
    for (int l = 0; l <= d.maxdepth; ++l) {
        d.level_off[l] = (int)flat.size();
        flat.insert(flat.end(), d.levels[l].begin(), d.levels[l].end());
    }
    d.level_off[d.maxdepth + 1] = (int)flat.size();
    if (d.d_tree) cudaFree(d.d_tree);
    if (d.d_levels) cudaFree(d.d_levels);
    cudaMalloc(&d.d_tree, sizeof(TreeNode) * d.T);
    cudaMalloc(&d.d_levels, sizeof(int) * flat.size());
    cudaMemcpy(d.d_tree, d.tree.data(), sizeof(TreeNode) * d.T, cudaMemcpyHostToDevice);
    cudaMemcpy(d.d_levels, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice);
    if (d.d_fr) cudaFree(d.d_fr);
    cudaMalloc(&d.d_fr, sizeof(FrontInfo) * d.T);
    d.built_for = e.cutoff;
}

int ensure_host_buf(Direct &d, int count)
{
    if (count <= d.h_buf_cap) return 0;
    if (d.h_buf) cudaFreeHost(d.h_buf);
    d.h_buf = nullptr;
    if (cudaMallocHost(&d.h_buf, sizeof(int) * count) != cudaSuccess) return SDDDST_ERR_NOMEM;
    d.h_buf_cap = count;
    return 0;
}

} // namespace

// ------------------------------------------------------------ host entry points

void direct_free(Engine &e)
{
    Direct *d = D(e);
    if (!d) return;
    void *bufs[] = {d->d_tree, d->d_tn, d->d_lrank, d->d_ctab, d->d_cnt, d->d_pos, d->d_own, d->d_perm, d->d_ucnt,
                    d->d_xw, d->d_yw, d->d_Y, d->d_upd, d->d_updpos, d->d_map, d->d_fr, d->d_levels, d->d_F,
                    d->d_inv, d->d_W, d->d_npert, d->d_Ff};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (d->h_buf) cudaFreeHost(d->h_buf);
    if (d->side) {
        cudaStreamSynchronize(d->side);
        cudaStreamDestroy(d->side);
    }
    for (cudaEvent_t ev : {d->ev_side, d->ev_next, d->ev_level})
        if (ev) cudaEventDestroy(ev);
    delete d;
    e.direct = nullptr;
}

// Symbolic phase for the Jacobian pattern assembled at positions x: the
// elimination order and each front's index set.
int direct_analyse(Engine &e, const double *x)
{
    if (!e.direct) {
        Direct *d = new Direct();
        e.direct = d;
        const int n = e.n;
        d->nchunk = (n + kChunk - 1) / kChunk;
        bool ok = cudaMalloc(&d->d_tn, sizeof(int) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_lrank, sizeof(int) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_pos, sizeof(int) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_own, sizeof(int) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_perm, sizeof(int) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_xw, sizeof(double) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_yw, sizeof(double) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_Y, sizeof(double) * n) == cudaSuccess &&
                  cudaMalloc(&d->d_npert, 2 * sizeof(int)) == cudaSuccess; // perturbed pivots, tensor-core failures
        if (!ok) {
            e.err = "direct solver: out of device memory";
            return SDDDST_ERR_NOMEM;
        }
    }
    Direct &d = *D(e);
    const int n = e.n;
    cudaStream_t st = e.st;
    if (d.built_for != e.cutoff) {
        build_tree(d, e);
        if (d.d_ctab) cudaFree(d.d_ctab);
        if (d.d_cnt) cudaFree(d.d_cnt);
        if (d.d_ucnt) cudaFree(d.d_ucnt);
        d.d_ctab = d.d_cnt = d.d_ucnt = nullptr;
        if (cudaMalloc(&d.d_ctab, sizeof(int) * (size_t)d.nchunk * d.T) != cudaSuccess ||
            cudaMalloc(&d.d_cnt, sizeof(int) * d.T) != cudaSuccess ||
            cudaMalloc(&d.d_ucnt, sizeof(int) * d.T) != cudaSuccess) {
            e.err = "direct solver: out of device memory";
            return SDDDST_ERR_NOMEM;
        }
    }
    d.analysed = d.factored = false;
    const int T = d.T;
    if (int rc = ensure_host_buf(d, 2 * T + 4)) {
        e.err = "direct solver: pinned buffer";
        return rc;
    }
    // 1) tree node of every dislocation, its rank inside its node
    assign_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, x, e.d_y, d.d_tree, d.d_tn, d.d_xw, d.d_yw);
    cudaMemsetAsync(d.d_ctab, 0, sizeof(int) * (size_t)d.nchunk * T, st);
    chunk_rank_kernel<<<d.nchunk, kChunk, 0, st>>>(n, T, d.d_tn, d.d_lrank, d.d_ctab);
    chunk_scan_kernel<<<(T + 255) / 256, 256, 0, st>>>(T, d.nchunk, d.d_ctab, d.d_cnt);
    cudaMemcpyAsync(d.h_buf, d.d_cnt, sizeof(int) * T, cudaMemcpyDeviceToHost, st);
    e.launches += 3;
    if (int rc = e.sync_check("direct analyse (counts)")) return rc;
    d.fr.assign(T, FrontInfo{});
    int start = 0;
    for (int t : d.postorder) {
        FrontInfo &f = d.fr[t];
        f.p = d.h_buf[t];
        f.start = start;
        start += f.p;
        f.parent = d.tree[t].parent;
        f.child0 = d.tree[t].child0;
        f.child1 = d.tree[t].child1;
        f.depth = d.tree[t].depth;
    }
    cudaMemcpyAsync(d.d_fr, d.fr.data(), sizeof(FrontInfo) * T, cudaMemcpyHostToDevice, st);
    place_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, T, d.d_tn, d.d_lrank, d.d_ctab, d.d_fr, d.d_pos, d.d_own);
    // 2) update sets
    update_set_kernel<false><<<T, 256, 0, st>>>(d.d_tree, d.d_fr, d.d_own, d.d_xw, d.d_yw, d.w, d.d_ucnt, nullptr,
                                                nullptr);
    cudaMemcpyAsync(d.h_buf, d.d_ucnt, sizeof(int) * T, cudaMemcpyDeviceToHost, st);
    e.launches += 2;
    if (int rc = e.sync_check("direct analyse (update sets)")) return rc;
    long uoff = 0, foff = 0, ioff = 0, woff = 0;
    double flops = 0.0;
    for (int t = 0; t < T; ++t) {
        FrontInfo &f = d.fr[t];
        f.u = d.h_buf[t];
        f.n = f.p + f.u;
        f.ld = (f.n + 1) & ~1;
        f.uoff = (int)uoff;
        f.foff = foff;
        f.ioff = ioff;
        f.woff = woff;
        uoff += f.u;
        foff += (long)f.n * f.ld;
        foff = (foff + 3) & ~3L;
        ioff += (long)((f.p + kNB - 1) / kNB) * 2 * kNB * kNB;
        woff += f.n;
        for (int k = 0; k < f.p; ++k) {
            const double r = (double)(f.n - k - 1);
            flops += r + 2.0 * r * r;
        }
    }
    if (uoff > 0x7fffffffL) {
        e.err = "direct solver: update lists exceed 2^31 entries";
        return SDDDST_ERR_CAPACITY;
    }
    d.flops = flops;
    d.F_used = foff;
    if (grow(d.d_upd, d.upd_cap, uoff) || grow(d.d_updpos, d.updpos_cap, uoff) || grow(d.d_map, d.map_cap, uoff)) {
        e.err = "direct solver: out of device memory (update lists)";
        return SDDDST_ERR_NOMEM;
    }
    d.f32 = e.prm.solver == SDDDST_SOLVER_DIRECT_MIXED;
    if ((d.f32 ? grow(d.d_Ff, d.Ff_cap, foff) : grow(d.d_F, d.F_cap, foff)) || grow(d.d_inv, d.inv_cap, ioff) ||
        grow(d.d_W, d.W_cap, woff)) {
        e.err = "direct solver: out of device memory (fronts)";
        return SDDDST_ERR_NOMEM;
    }
    const int L = d.maxdepth + 1;
    d.level_pmax.assign(L, 0);
    d.level_nmax.assign(L, 0);
    d.level_umax.assign(L, 0);
    for (int l = 0; l < L; ++l)
        for (int t : d.levels[l]) {
            d.level_pmax[l] = std::max(d.level_pmax[l], d.fr[t].p);
            d.level_nmax[l] = std::max(d.level_nmax[l], d.fr[t].n);
            for (int c : {d.fr[t].child0, d.fr[t].child1})
                if (c >= 0) d.level_umax[l] = std::max(d.level_umax[l], d.fr[c].u);
        }
    cudaMemcpyAsync(d.d_fr, d.fr.data(), sizeof(FrontInfo) * T, cudaMemcpyHostToDevice, st);
    update_set_kernel<true><<<T, 256, 0, st>>>(d.d_tree, d.d_fr, d.d_own, d.d_xw, d.d_yw, d.w, nullptr, d.d_upd,
                                               d.d_updpos);
    cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
    map_kernel<<<T, 256, 0, st>>>(T, d.d_fr, d.d_updpos, d.d_map, e.d_flag);
    e.launches += 2;
    cudaMemcpyAsync(&d.h_buf[0], e.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("direct analyse (maps)")) return rc;
    if (d.h_buf[0]) {
        e.err = "direct solver: a child's update set is not inside its parent's front";
        return SDDDST_ERR_CAPACITY;
    }
    d.analysed = true;
    return 0;
}

// Numeric factorization of J(h) = I + diag((1 + d)/2) h G on the analysed
// pattern, into FP64 or FP32 fronts.
template <typename FT> static int factor_impl(Engine &e, Direct &d, double h, const double *dvec, FT *F)
{
    cudaStream_t st = e.st;
    cudaFuncSetAttribute(diag_block_kernel<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem);
    cudaFuncSetAttribute(panel_kernel<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem);
    cudaFuncSetAttribute(update_kernel<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem<FT>());
    if (!d.side) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (cudaStreamCreateWithPriority(&d.side, cudaStreamNonBlocking, greatest) != cudaSuccess ||
            cudaEventCreateWithFlags(&d.ev_side, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&d.ev_next, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&d.ev_level, cudaEventDisableTiming) != cudaSuccess) {
            e.err = "direct solver: stream or event creation failed";
            return SDDDST_ERR_CUDA;
        }
    }
    cudaMemsetAsync(F, 0, sizeof(FT) * (size_t)d.F_used, st);
    cudaMemsetAsync(e.d_flag, 0, sizeof(int), st);
    cudaMemsetAsync(d.d_npert, 0, 2 * sizeof(int), st);
    // FP32 fronts: the trailing updates on the CUDA cores by default; with
    // SDDDST_LU_TENSOR_CORES set, on the tensor cores (compensated TF32).  At
    // N = 16384 (31 fronts) the tensor-core updates take 17.4 ms per
    // factorization against 11.9 ms on the CUDA cores: each 32-deep K chunk
    // is 12 short MMAs behind a register-staged split of A and B into their
    // TF32 high and low parts, which the CTA's 128 threads cannot hide.
    const int *list_cur = nullptr;
    const bool tc = sizeof(FT) == 4 && std::getenv("SDDDST_LU_TENSOR_CORES") != nullptr;
    if (tc) cudaFuncSetAttribute(update_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    auto update = [&](unsigned gx, int nf_, cudaStream_t s_, int J_, int mode) {
        if (tc)
            update_tc_kernel<<<dim3(gx, nf_), 128, kTcSmem, s_>>>(d.d_fr, list_cur, J_, mode,
                                                                 reinterpret_cast<float *>(F), d.d_npert + 1);
        else
            update_kernel<FT><<<dim3(gx, nf_), 256, upd_smem<FT>(), s_>>>(d.d_fr, list_cur, J_, mode, F);
    };
    const int wpb = 8;
    if (e.valf)
        assemble_kernel<float, FT><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(
            e.n, h, e.d_rowptr, e.d_col, e.d_valf, e.d_gdiag, dvec, d.d_tn, d.d_pos, d.d_fr, d.d_updpos, F,
            e.d_flag);
    else
        assemble_kernel<double, FT><<<(e.n + wpb - 1) / wpb, 32 * wpb, 0, st>>>(
            e.n, h, e.d_rowptr, e.d_col, e.d_val, e.d_gdiag, dvec, d.d_tn, d.d_pos, d.d_fr, d.d_updpos, F,
            e.d_flag);
    e.launches++;
    for (int l = d.maxdepth; l >= 0; --l) {
        const int nf = (int)d.levels[l].size();
        const int *list = d.d_levels + d.level_off[l];
        list_cur = list;
        if (d.level_umax[l] > 0) {
            const int tiles = (d.level_umax[l] + 31) / 32;
            for (int slot = 0; slot < 2; ++slot)
                extend_add_kernel<FT><<<dim3(tiles * tiles, nf), 256, 0, st>>>(d.d_fr, list, slot, F, d.d_map);
            e.launches += 2;
        }
        // outer blocks of 128 pivots: two pivot blocks of 64, the trailing
        // update once per outer block (K = 128).  The side stream factors
        // outer block J's pivot blocks (they need only the columns of J that
        // outer block J-1's mode-2 update produced) while the main stream
        // still updates the rest of the trailing matrix (mode 3 of J-1).
        cudaEventRecord(d.ev_level, st);
        cudaStreamWaitEvent(d.side, d.ev_level, 0);
        const int nouter = (d.level_pmax[l] + 2 * kNB - 1) / (2 * kNB);
        for (int J = 0; J < nouter; ++J) {
            const int j0 = 2 * J, j1 = j0 + 1;
            const int rest = std::max(1, d.level_nmax[l] - J * 2 * kNB); // bounds every row / column count below
            const int half = (rest + kNB - 1) / kNB;
            const int tiles = (rest + kBM - 1) / kBM;
            if (J > 0) cudaStreamWaitEvent(d.side, d.ev_next, 0);
            diag_block_kernel<FT><<<dim3(1, nf), kDiagThreads, kDiagSmem, d.side>>>(d.d_fr, list, j0, F, d.d_inv,
                                                                                d.d_perm, d.d_npert);
            panel_kernel<FT><<<dim3(1 + half, nf), 256, kPanelSmem, d.side>>>(d.d_fr, list, j0, F, d.d_inv,
                                                                         d.d_perm, 1, 1, 1);
            update(tiles, nf, d.side, J, 0);
            diag_block_kernel<FT><<<dim3(1, nf), kDiagThreads, kDiagSmem, d.side>>>(d.d_fr, list, j1, F, d.d_inv,
                                                                                d.d_perm, d.d_npert);
            cudaEventRecord(d.ev_side, d.side);
            cudaStreamWaitEvent(st, d.ev_side, 0);
            panel_kernel<FT><<<dim3(half, nf), 256, kPanelSmem, st>>>(d.d_fr, list, j0, F, d.d_inv, d.d_perm, 2,
                                                                 half, 0);
            update(tiles, nf, st, J, 1);
            panel_kernel<FT><<<dim3(2 * half, nf), 256, kPanelSmem, st>>>(d.d_fr, list, j1, F, d.d_inv, d.d_perm,
                                                                     3, half, 1);
            update(2 * tiles, nf, st, J, 2);
            cudaEventRecord(d.ev_next, st);
            update(tiles * tiles, nf, st, J, 3);
            e.launches += 9;
        }
    }
    int hv[3];
    cudaMemcpyAsync(&d.h_buf[0], e.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&d.h_buf[1], d.d_npert, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int rc = e.sync_check("direct factor")) return rc;
    hv[0] = d.h_buf[0];
    hv[1] = d.h_buf[1];
    hv[2] = d.h_buf[2];
    if (hv[2]) {
        e.err = "direct solver: a tensor-core update did not complete";
        return SDDDST_ERR_CUDA;
    }
    if (hv[0]) {
        e.err = "direct solver: a Jacobian entry falls outside its front";
        return SDDDST_ERR_CAPACITY;
    }
    d.perturbed += hv[1];
    d.factorizations++;
    d.factored = true;
    return 0;
}


int direct_factor(Engine &e, double h, const double *dvec)
{
    Direct *dp = D(e);
    if (!dp || !dp->analysed) {
        e.err = "direct solver: factorization before analysis";
        return SDDDST_ERR_INVALID;
    }
    return dp->f32 ? factor_impl<float>(e, *dp, h, dvec, dp->d_Ff) : factor_impl<double>(e, *dp, h, dvec, dp->d_F);
}

// x = (LU)^-1 b with the current factors; b and x may alias.
template <typename FT> static int apply_impl(Engine &e, Direct &d, const double *b, double *x, const FT *F)
{
    cudaStream_t st = e.st;
    for (int l = d.maxdepth; l >= 0; --l) {
        const int nf = (int)d.levels[l].size();
        const int *list = d.d_levels + d.level_off[l];
        fgather_kernel<<<nf, 256, 0, st>>>(d.d_fr, list, d.d_own, d.d_map, b, d.d_W);
        const int nblk = (d.level_pmax[l] + kNB - 1) / kNB;
        for (int j = 0; j < nblk; ++j) {
            const int rest = std::max(1, d.level_nmax[l] - j * kNB);
            fblock_kernel<FT><<<dim3((rest + kRowsPerCta - 1) / kRowsPerCta, nf), 256, 0, st>>>(
                d.d_fr, list, j, F, d.d_inv, d.d_perm, d.d_W, d.d_Y);
        }
        e.launches += 1 + nblk;
    }
    for (int l = 0; l <= d.maxdepth; ++l) {
        const int nf = (int)d.levels[l].size();
        const int *list = d.d_levels + d.level_off[l];
        const int pm = d.level_pmax[l];
        if (pm == 0) continue;
        bupdate_kernel<FT><<<dim3((pm + kRowsPerCta - 1) / kRowsPerCta, nf), 256, 0, st>>>(d.d_fr, list, F, d.d_upd,
                                                                                    d.d_Y, x, d.d_W);
        const int nblk = (pm + kNB - 1) / kNB;
        for (int j = nblk - 1; j >= 0; --j) {
            const int rows = std::max(1, j * kNB);
            bblock_kernel<FT><<<dim3((rows + kRowsPerCta - 1) / kRowsPerCta, nf), 256, 0, st>>>(
                d.d_fr, list, j, F, d.d_inv, d.d_own, d.d_W, x);
        }
        e.launches += 1 + nblk;
    }
    return 0;
}


int direct_apply(Engine &e, const double *b, double *x)
{
    Direct *dp = D(e);
    if (!dp || !dp->factored) {
        e.err = "direct solver: solve before factorization";
        return SDDDST_ERR_INVALID;
    }
    return dp->f32 ? apply_impl<float>(e, *dp, b, x, dp->d_Ff) : apply_impl<double>(e, *dp, b, x, dp->d_F);
}

// Direct solve refined against the unfactored J: refinement steps on the
// FP64 residual (up to 3 with FP64 factors, 10 with FP32 factors, which gain
// about cond(J) * 6e-8 per step), then GMRES preconditioned by the factors.
int direct_solve(Engine &e, double h, const double *dvec, const double *rhs, double *x)
{
    const int n = e.n;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const double tol = e.prm.solver_tol > 0 ? e.prm.solver_tol : 1e-13;
    double bn2 = 0.0;
    if (int rc = e.sum_sq(rhs, &bn2)) return rc;
    if (!std::isfinite(bn2)) {
        e.err = "solve: non-finite right-hand side";
        return SDDDST_ERR_NONFINITE;
    }
    e.solves++;
    if (bn2 == 0.0) {
        cudaMemsetAsync(x, 0, sizeof(double) * n, e.st);
        e.last_iters = 0;
        return 0;
    }
    if (int rc = direct_apply(e, rhs, x)) return rc;
    const int max_ref = D(e)->f32 ? 10 : 3;
    for (int it = 0; it <= max_ref; ++it) {
        launch_spmv_J(e, h, dvec, x, e.d_w, e.st);
        resid_kernel<<<nb, 256, 0, e.st>>>(n, rhs, e.d_w, e.d_r);
        e.launches++;
        double rn2 = 0.0;
        if (int rc = e.sum_sq(e.d_r, &rn2)) return rc;
        if (!std::isfinite(rn2)) break;
        e.last_resid = std::sqrt(rn2 / bn2);
        if (rn2 <= tol * tol * bn2) {
            e.last_iters = it;
            e.iterations += it;
            return 0;
        }
        if (it == max_ref) break;
        if (int rc = direct_apply(e, e.d_r, e.d_z)) return rc;
        addto_kernel<<<nb, 256, 0, e.st>>>(n, e.d_z, x);
        e.launches++;
    }
    e.stalls++;
    e.solves--; // counted again by GMRES
    return gmres_solve(e, h, dvec, rhs, x, 3);
}

int direct_stats(const Engine &e, long *factorizations, long *perturbed, double *flops, long *front_doubles,
                 int *fronts, int *depth)
{
    const Direct *d = static_cast<const Direct *>(e.direct);
    if (!d) {
        *factorizations = *perturbed = *front_doubles = 0;
        *flops = 0.0;
        *fronts = *depth = 0;
        return 0;
    }
    *factorizations = d->factorizations;
    *perturbed = d->perturbed;
    *flops = d->flops;
    *front_doubles = d->F_used;
    *fronts = d->T;
    *depth = d->maxdepth + 1;
    return 0;
}

} // namespace sd
