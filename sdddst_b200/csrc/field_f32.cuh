// FP32 field kernel for the mixed-precision pair sum.
//
// Same image structure as field_f64.cuh (AnalyticField.cpp:145-160): the
// separation is formed and wrapped in FP64 (so close pairs keep full relative
// accuracy) and rounded to FP32 once; the image terms run in FP32 with the
// SFU (ex2, rcp); the caller accumulates the per-pair results in FP64.
//  * k = 0 uses cosh 2a - cos 2b = 2(sinh^2 a + sin^2 b) and
//    cosh 2a cos 2b - 1 = 2(sinh^2 a - sin^2 b) - 4 sinh^2 a sin^2 b, with
//    sinh a from its odd Taylor series below |a| = 0.5 (truncation < 4e-9
//    relative) and from e^{+-a} above;
//  * |k| = 1 images are exact: (C cy - 1) / (C - cy)^2 with C = cosh 2pi u;
//  * |u| >= 1.5 images use t = 1/C = 2 e^{-2 pi |u|} (the dropped e^{-4 pi |u|}
//    part is below 7e-9 relative) and N/D^2 = cy t + (2 cy^2 - 1) t^2 +
//    O(t^3) (|t| <= 1.6e-4, so the remainder is below 3e-8 relative), which
//    needs neither a division nor an SFU op.
#pragma once

#include "common.cuh"

namespace sd {

constexpr float kPiF = 3.14159265358979f;
constexpr float kTwoPiSqF = 19.7392088021787f;

// e^{-2 pi k} in FP32, k = 1..5
__device__ __forceinline__ float qnegf(int k)
{
    switch (k) {
    case 1: return 1.8674427317079889e-03f;
    case 2: return 3.4873423562089956e-06f;
    case 3: return 6.512412136079901e-09f;
    case 4: return 1.2161556709409309e-11f;
    default: return 2.2711010683240937e-14f;
    }
}
__device__ __forceinline__ float qposf(int k)
{
    switch (k) {
    case 1: return 535.4916555247647f;
    case 2: return 286751.3131366533f;
    case 3: return 153552935.3954467f;
    case 4: return 82226315585.595f;
    default: return 44031505860632.03f;
    }
}

__device__ __forceinline__ float sinh_small_or_exp(float a, float ep, float epi)
{
    float a2 = a * a;
    float poly = a * (1.0f + a2 * (1.0f / 6.0f + a2 * (1.0f / 120.0f + a2 * (1.0f / 5040.0f))));
    return fabsf(a) < 0.5f ? poly : 0.5f * (ep - epi);
}

// tau_xy(dx, dy) in FP32 from FP64 separations.
__device__ __forceinline__ float tau_xy_f32(double dxd, double dyd)
{
    const float dx = (float)dxd, dy = (float)dyd;
    const float sn = sinpif(dy);
    const float sn2 = sn * sn;
    const float cy = 1.0f - 2.0f * sn2;
    const float a = kPiF * dx;
    const float ep = __expf(a);
    const float epi = __expf(-a);
    const float sh = sinh_small_or_exp(a, ep, epi);
    const float sh2 = sh * sh;
    const float E = ep * ep, Ei = epi * epi;
    const bool pos = dx >= 0.0f;

    // k = 0
    const float D0 = 2.0f * (sh2 + sn2);
    const float N0 = 2.0f * (sh2 - sn2) - 4.0f * sh2 * sn2;
    const float r0 = __frcp_rn(D0);
    float acc = dx * N0 * r0 * r0;

    // |k| = 1, exact
    {
        float Cp = 0.5f * (E * qposf(1) + Ei * qnegf(1));
        float Dp = Cp - cy;
        float rp = __frcp_rn(Dp * Dp);
        float Cm = 0.5f * (E * qnegf(1) + Ei * qposf(1));
        float Dm = Cm - cy;
        float rm = __frcp_rn(Dm * Dm);
        acc += (dx + 1.0f) * (Cp * cy - 1.0f) * rp + (dx - 1.0f) * (Cm * cy - 1.0f) * rm;
    }
    // far images: t = 2 e^{-2 pi |u|}
    const float c2 = 2.0f * cy * cy - 1.0f;
    float far = 0.0f;
#pragma unroll
    for (int k = 2; k <= 4; ++k) {
        float tp = 2.0f * Ei * qnegf(k); // u = dx + k > 0
        float tm = 2.0f * E * qnegf(k);  // u = dx - k < 0
        float wp = (k == 4 && pos) ? 1.0f - dx : 1.0f;
        float wm = (k == 4 && !pos) ? 1.0f + dx : 1.0f;
        far += wp * (dx + (float)k) * tp * (cy + c2 * tp) + wm * (dx - (float)k) * tm * (cy + c2 * tm);
    }
    {
        float t5 = pos ? 2.0f * E * qnegf(5) : 2.0f * Ei * qnegf(5);
        float u5 = pos ? dx - 5.0f : dx + 5.0f;
        far += fabsf(dx) * u5 * t5 * (cy + c2 * t5);
    }
    return (acc + far) * kTwoPiSqF;
}

} // namespace sd
