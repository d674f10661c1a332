// Shared device helpers of the sdddst_b200 engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

namespace sd {

constexpr double kPi = 3.141592653589793115997963468544185161590576171875;
constexpr double kTwoPiSq = 0x1.3bd3cc9be45dep+4; // 2*pi^2
constexpr double kEps = 1e-12;                     // EPS, reference include/constants.h:24

// e^{2 pi k} and e^{-2 pi k}, k = 0..5, correctly rounded.
__device__ __forceinline__ double qpos(int k)
{
    switch (k) {
    case 1: return 0x1.0bbeee9177e19p+9;
    case 2: return 0x1.1807d40a6e514p+18;
    case 3: return 0x1.24e104eca77fdp+27;
    case 4: return 0x1.3251201419852p+36;
    case 5: return 0x1.405f122040c04p+45;
    default: return 1.0;
    }
}
__device__ __forceinline__ double qneg(int k)
{
    switch (k) {
    case 1: return 0x1.e989f5d6dff5cp-10;
    case 2: return 0x1.d4102bc3f7d4cp-19;
    case 3: return 0x1.bf8790de8c93cp-28;
    case 4: return 0x1.abe59085010e2p-37;
    case 5: return 0x1.99200ce920dfap-46;
    default: return 1.0;
    }
}

// Minimum image into [-0.5, 0.5): the reference's normalize() loop
// (include/utility.h:29-40).  Every subtraction of 1 is exact below 2^53, so
// shifting large |v| by floor(v) first gives bit-identical results while
// bounding the loop; non-finite values are returned unchanged instead of
// looping forever.
__device__ __forceinline__ double wrap_half(double v)
{
    if (!(fabs(v) < 8.0)) {
        if (!isfinite(v)) return v;
        v -= floor(v);
    }
    while (v < -0.5) v += 1.0;
    while (v >= 0.5) v -= 1.0;
    return v;
}

// r^2 = dx*dx + dy*dy rounded as the reference computes it on the host
// (two products and a sum, no fused multiply-add), so decisions taken on it
// (tolerances, cutoff pattern) match bit for bit.
__device__ __forceinline__ double r2_exact(double dx, double dy)
{
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Non-negative doubles order like their bit patterns: atomicMin on the bits.
__device__ __forceinline__ void atomic_min_nonneg(unsigned long long *addr, double v)
{
    atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

} // namespace sd
