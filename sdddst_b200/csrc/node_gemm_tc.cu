// Node-level products of the learned preconditioner's network on the 5th-gen
// tensor cores (tcgen05): for a tile of 128 nodes,
//   D[128 x NOUT] = X[128 x K] W[NOUT x K]^T
// with X the node states rounded to BF16, W the BF16 weights (PyTorch's
// [out][in] layout, i.e. K-major) and D accumulated in FP32 in tensor memory.
// Two forms (sdddst_b200/learned.py, Net.forward):
//   kProj:   X = h (K = 64), W = [P; Q] (NOUT = 128):  ph = D[:, :64] + b_P
//            (FP32), qh = D[:, 64:] (stored in BF16, the edge pass's gather);
//   kUpdate: X = [h; a] (K = 128), W = U (NOUT = 64):   h += relu(D + b_U).
// One CTA of 128 threads per tile: the threads stage both operands in shared
// memory in the no-swizzle K-major core-matrix layout (8 rows x 16 bytes per
// 128-byte core matrix; K-adjacent core matrices 128 bytes apart, 8-row groups
// K/8 x 128 bytes apart), one thread issues the K/16 MMAs
// (tcgen05.mma.cta_group::1.kind::f16, M = 128) and commits them to an
// mbarrier, every warp then reads its 32 TMEM lanes (its 32 nodes) with
// tcgen05.ld and applies the epilogue.  The mbarrier wait is bounded: past
// its limit the kernel records the failure in *err and skips the read; the
// tensor memory is released on every path.  No TMA and no cluster: a
// single-CTA kernel over this GPU's own memory.
#include <cuda_bf16.h>

#include "engine.h"

namespace sd {

namespace {

constexpr int kTileM = 128;

// byte offset of element (r, k) of an R x K BF16 tile (layout above)
__device__ __forceinline__ unsigned cm_offset(int r, int k, int K)
{
    return (unsigned)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading-dimension byte
// offset (between K-adjacent core matrices), stride byte offset (between
// 8-row groups), descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned pack_bf16x2(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b); // .x = a (low half), .y = b
    return *reinterpret_cast<const unsigned *>(&v);
}

enum { kProj = 0, kUpdate = 1 };

template <int MODE>
struct Shape;
template <>
struct Shape<kProj> {
    static constexpr int K = 64, NOUT = 128;
};
template <>
struct Shape<kUpdate> {
    static constexpr int K = 128, NOUT = 64;
};

template <int MODE>
__global__ void __launch_bounds__(128) node_gemm_tc_kernel(int n, float *__restrict__ xa,
                                                           const float *__restrict__ xb,
                                                           const __nv_bfloat16 *__restrict__ w, long oW0, long oW1,
                                                           long oBias, float *__restrict__ out_f,
                                                           __nv_bfloat16 *__restrict__ out_h, int *__restrict__ err)
{
    constexpr int K = Shape<MODE>::K, NOUT = Shape<MODE>::NOUT;
    constexpr unsigned kSBO = (K / 8) * 128, kLBO = 128;
    constexpr unsigned kCols = NOUT; // TMEM columns: one FP32 accumulator column per output channel
    // instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
    // N = NOUT, M = 128
    constexpr unsigned kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(NOUT >> 3) << 17) |
                                ((unsigned)(kTileM >> 4) << 24);
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char *As = tc_smem;                  // 128 x K BF16
    unsigned char *Bs = tc_smem + kTileM * K * 2; // NOUT x K BF16
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = blockIdx.x * kTileM;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    // A: thread tid stages node row tid (zeros past n), eight K values per
    // 16-byte store
    {
        const int r = tid, i = i0 + r;
#pragma unroll
        for (int k8 = 0; k8 < K / 8; ++k8) {
            float v[8];
            const float *src = (MODE == kUpdate && k8 >= 8) ? xb : xa;
            const int kk = (MODE == kUpdate && k8 >= 8) ? 8 * (k8 - 8) : 8 * k8;
            if (i < n) {
                const float4 a = *reinterpret_cast<const float4 *>(src + (long)i * 64 + kk);
                const float4 b = *reinterpret_cast<const float4 *>(src + (long)i * 64 + kk + 4);
                v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
                v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] = 0.0f;
            }
            uint4 p;
            p.x = pack_bf16x2(v[0], v[1]);
            p.y = pack_bf16x2(v[2], v[3]);
            p.z = pack_bf16x2(v[4], v[5]);
            p.w = pack_bf16x2(v[6], v[7]);
            *reinterpret_cast<uint4 *>(As + cm_offset(r, 8 * k8, K)) = p;
        }
    }
    // B: the weights, element by element (the flat weight array has no
    // alignment guarantee beyond 2 bytes)
    {
        const unsigned short *wb = reinterpret_cast<const unsigned short *>(w);
        for (int idx = tid; idx < NOUT * K; idx += blockDim.x) {
            const int c = idx / K, k = idx % K;
            unsigned short bits;
            if (MODE == kProj) bits = c < 64 ? wb[oW0 + (long)c * K + k] : wb[oW1 + (long)(c - 64) * K + k];
            else bits = wb[oW0 + (long)c * K + k];
            *reinterpret_cast<unsigned short *>(Bs + cm_offset(c, k, K)) = bits;
        }
    }
    // the generic-proxy stores become visible to the tensor cores' async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_slot;
    if (tid == 0) {
        const unsigned a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
        for (int t = 0; t < K / 16; ++t) {
            const unsigned long long ad = smem_desc(a0 + 256u * t, kLBO, kSBO);
            const unsigned long long bd = smem_desc(b0 + 256u * t, kLBO, kSBO);
            const unsigned acc = t > 0 ? 1u : 0u;
            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                         "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
    }
    // bounded wait for the MMAs' completion (phase 0 of the mbarrier)
    unsigned done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(smem_u32(&mbar)), "r"(0u)
                     : "memory");
        if (!done && it > 32) __nanosleep(64);
    }
    if (!done && lane == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // `done` is the mbarrier's phase, the same for every thread; a warp that
    // gave up skips the warp-wide load
    if (__all_sync(0xffffffffu, done)) {
        const int r = warp * 32 + lane, i = i0 + r;
        const unsigned lane_base = (unsigned)(warp * 32) << 16;
#pragma unroll
        for (int c0 = 0; c0 < NOUT; c0 += 16) {
            unsigned v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + lane_base + (unsigned)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (i < n) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int c = c0 + q;
                    const float d = __uint_as_float(v[q]);
                    if (MODE == kProj) {
                        if (c < 64) out_f[(long)i * 64 + c] = d + __bfloat162float(w[oBias + c]);
                        else out_h[(long)i * 64 + c - 64] = __float2bfloat16_rn(d);
                    } else {
                        const float u = d + __bfloat162float(w[oBias + c]);
                        xa[(long)i * 64 + c] += fmaxf(u, 0.0f);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// Both forms request 48 KB of shared memory (the projection needs 32 KB):
// at most four CTAs fit on an SM, so their tensor memory (at most 128
// columns each) never exceeds the SM's 512 columns and no allocation waits.
template <int MODE>
constexpr size_t tc_smem_bytes()
{
    static_assert((kTileM + Shape<MODE>::NOUT) * Shape<MODE>::K * 2 <= 48 * 1024, "operand tiles exceed 48 KB");
    return 48 * 1024;
}

// 48 KB of dynamic shared memory beside the kernel's static barrier words
// needs the opt-in above 48 KB per block (set once per device)
void set_smem_attr()
{
    static bool done[256] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev > 255 || done[dev]) return;
    cudaFuncSetAttribute(node_gemm_tc_kernel<kProj>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(node_gemm_tc_kernel<kUpdate>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    done[dev] = true;
}

} // namespace

// ph = P h + b_P (FP32), qh = Q h (BF16) for all n nodes
void launch_node_proj_tc(int n, const float *h, const __nv_bfloat16 *w, long oP, long oPb, long oQ, float *ph,
                         __nv_bfloat16 *qh, int *err, cudaStream_t st)
{
    set_smem_attr();
    node_gemm_tc_kernel<kProj><<<(unsigned)((n + kTileM - 1) / kTileM), 128, tc_smem_bytes<kProj>(), st>>>(
        n, const_cast<float *>(h), nullptr, w, oP, oQ, oPb, ph, qh, err);
}

// h += relu(U [h; a] + b_U) for all n nodes
void launch_node_update_tc(int n, float *h, const float *a, const __nv_bfloat16 *w, long oU, long oUb, int *err,
                           cudaStream_t st)
{
    set_smem_attr();
    node_gemm_tc_kernel<kUpdate><<<(unsigned)((n + kTileM - 1) / kTileM), 128, tc_smem_bytes<kUpdate>(), st>>>(
        n, h, a, w, oU, 0, oUb, nullptr, nullptr, err);
}

} // namespace sd
