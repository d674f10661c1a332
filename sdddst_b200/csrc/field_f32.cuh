// FP32 field kernel for the mixed-precision pair sum.
//
// Same image structure as field_f64.cuh (AnalyticField.cpp:145-160).  The
// separation is formed and wrapped in FP64 by the caller (so close pairs keep
// full relative accuracy) and rounded to FP32 once; the image terms run in
// FP32 with the SFU (ex2, rcp); the caller accumulates in FP64.
//  * sin(pi dy), |dy| <= 0.5, is an odd degree-13 polynomial (Taylor; the
//    remainder is below 7e-10);
//  * k = 0 uses cosh 2a - cos 2b = 2(sinh^2 a + sin^2 b) and
//    cosh 2a cos 2b - 1 = 2(sinh^2 a - sin^2 b) - 4 sinh^2 a sin^2 b, with
//    sinh a from its odd Taylor series below |a| = 0.5 (remainder < 4e-9
//    relative) and from e^{+-a} above;
//  * |k| = 1 images are exact: (C cy - 1) / (C - cy)^2 with C = cosh 2pi u;
//  * |u| >= 1.5 images use t = 1/C = 2 e^{-2 pi |u|} (dropped part below
//    7e-9 relative) and N/D^2 = cy t + (2 cy^2 - 1) t^2 + O(t^3); with
//    t = 2 E^{-+1} e^{-2 pi k} the sums over k = 2..4 collapse to
//    polynomials in dx with constant coefficients (the t^2 part is kept for
//    k = 2 only; for k >= 3 it is below 3e-7 of a term that is itself below
//    1e-7 of tau);
//  * the reference's end image (weight |dx|, at |u| >= 4.5: below 5e-11 in
//    tau_xy) and the partial weight of the k = 4 image (below 1e-9) are left
//    out: both are far below the FP32 resolution of the sum.
#pragma once

#include "common.cuh"

namespace sd {

constexpr float kPiF = 3.14159265358979f;
constexpr float kTwoPiSqF = 19.7392088021787f;

// e^{+-2 pi k} and the far-image sums
constexpr float kQP1 = 535.4916555247647f;                       // e^{2 pi}
constexpr float kQN1 = 1.8674427317079889e-03f;                  // e^{-2 pi}
constexpr float kQN2 = 3.4873423562089956e-06f;
constexpr float kQN3 = 6.512412136079901e-09f;
constexpr float kA1 = 3.4938669795049805e-06f;                   // qn2 + qn3 + qn4
constexpr float kB1 = 6.994256639099779e-06f;                    // 2 qn2 + 3 qn3 + 4 qn4
constexpr float kQN2SQ = 1.2161556709409309e-11f;                // qn2^2 = qn4

// Single-instruction approximate reciprocal (SFU, about 1 ulp); the FP32
// path's accuracy target is set by its FP32 inputs, not by this rounding.
__device__ __forceinline__ float rcp_fast(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float sinpi_poly(float y)
{
    const float y2 = y * y;
    float p = 0.00046630280576761f;   //  pi^13 / 13!
    p = fmaf(p, y2, -0.00737043094571435f); // -pi^11 / 11!
    p = fmaf(p, y2, 0.08214588661112823f);  //  pi^9 / 9!
    p = fmaf(p, y2, -0.59926452932079207f); // -pi^7 / 7!
    p = fmaf(p, y2, 2.55016403987734549f);  //  pi^5 / 5!
    p = fmaf(p, y2, -5.16771278004997003f); // -pi^3 / 3!
    p = fmaf(p, y2, 3.14159265358979324f);  //  pi
    return y * p;
}

// tau_xy(dx, dy) in FP32; dx, dy already minimum-image in [-0.5, 0.5].
__device__ __forceinline__ float tau_xy_f32(float dx, float dy)
{
    const float sn = sinpi_poly(dy);
    const float sn2 = sn * sn;
    const float cy = fmaf(-2.0f, sn2, 1.0f);
    const float a = kPiF * dx;
    const float ep = __expf(a);
    const float epi = __expf(-a);
    const float a2 = a * a;
    const float poly = a * fmaf(a2, fmaf(a2, fmaf(a2, 1.0f / 5040.0f, 1.0f / 120.0f), 1.0f / 6.0f), 1.0f);
    const float sh = fabsf(a) < 0.5f ? poly : 0.5f * (ep - epi);
    const float sh2 = sh * sh;
    const float E = ep * ep, Ei = epi * epi;

    // k = 0
    const float D0 = 2.0f * (sh2 + sn2);
    const float N0 = fmaf(-4.0f * sh2, sn2, 2.0f * (sh2 - sn2));
    const float r0 = rcp_fast(D0);
    float acc = dx * N0 * r0 * r0;

    // |k| = 1, exact
    {
        const float Cp = 0.5f * fmaf(E, kQP1, Ei * kQN1);
        const float Dp = Cp - cy;
        const float rp = rcp_fast(Dp * Dp);
        const float Cm = 0.5f * fmaf(E, kQN1, Ei * kQP1);
        const float Dm = Cm - cy;
        const float rm = rcp_fast(Dm * Dm);
        acc = fmaf((dx + 1.0f) * fmaf(Cp, cy, -1.0f), rp, acc);
        acc = fmaf((dx - 1.0f) * fmaf(Cm, cy, -1.0f), rm, acc);
    }
    // |u| >= 1.5: first-order sums over k = 2..4 (+k side uses E^-1, -k side E)
    const float c2 = fmaf(2.0f * cy, cy, -1.0f);
    const float base = dx * kA1;
    float far = 2.0f * cy * fmaf(Ei, base + kB1, E * (base - kB1));
    far = fmaf(4.0f * c2 * kQN2SQ, fmaf(Ei * Ei, dx + 2.0f, E * E * (dx - 2.0f)), far);
    return (acc + far) * kTwoPiSqF;
}

} // namespace sd

namespace sd {

// d tau_xy / d dx in FP32 (the Jacobian of the mixed path), same image
// structure as tau_xy_dx_f64:  sum_k w_k f'(u_k) + sigma (f(u_end) - f(u_edge)),
//   f'(u) = 2 pi^2 / D^2 [N + 2 pi u S (cy - 2 N / D)]   (k = 0, +-1 exact);
// for |u| >= 1.5, t = 1/C = 2 e^{-2 pi |u|}:
//   f'(u) = 2 pi^2 [ (1 - 2 pi |u|) cy t
//                   + ((2 cy^2 - 1) + 2 pi |u| (2 - 4 cy^2)) t^2 ] + O(t^3),
//   f(u)  = 2 pi^2 u cy t + O(t^2),
// with the second order kept for k = 2 only and the k = 2..4 first-order sums
// collapsed to polynomials in dx.  The end image, the partial weight of the
// k = 4 image and the end/edge difference of the reference's weighting are
// left out (each below 1.2e-6 absolute, while |d tau / dx| >= 4 over the
// cell: below the FP32 resolution of the value).
__device__ __forceinline__ float tau_xy_dx_f32(float dx, float dy)
{
    const float twopi = 6.28318530717959f;
    const float sn = sinpi_poly(dy);
    const float sn2 = sn * sn;
    const float cy = fmaf(-2.0f, sn2, 1.0f);
    const float a = kPiF * dx;
    const float ep = __expf(a);
    const float epi = __expf(-a);
    const float a2 = a * a;
    const float poly = a * fmaf(a2, fmaf(a2, fmaf(a2, 1.0f / 5040.0f, 1.0f / 120.0f), 1.0f / 6.0f), 1.0f);
    const float sh = fabsf(a) < 0.5f ? poly : 0.5f * (ep - epi);
    const float ch = 0.5f * (ep + epi);
    const float sh2 = sh * sh;
    const float E = ep * ep, Ei = epi * epi;

    // k = 0
    const float D0 = 2.0f * (sh2 + sn2);
    const float N0 = fmaf(-4.0f * sh2, sn2, 2.0f * (sh2 - sn2));
    const float S0 = 2.0f * sh * ch;
    const float r0 = rcp_fast(D0);
    float acc = r0 * r0 * fmaf(twopi * dx * S0, fmaf(-2.0f * N0, r0, cy), N0);
    // |k| = 1
    {
        const float ap = E * kQP1, bp = Ei * kQN1;
        const float Cp = 0.5f * (ap + bp), Sp = 0.5f * (ap - bp);
        const float Dp = Cp - cy, Np = fmaf(Cp, cy, -1.0f);
        const float rp = rcp_fast(Dp);
        acc = fmaf(rp * rp, fmaf(twopi * (dx + 1.0f) * Sp, fmaf(-2.0f * Np, rp, cy), Np), acc);
        const float am = E * kQN1, bm = Ei * kQP1;
        const float Cm = 0.5f * (am + bm), Sm = 0.5f * (am - bm);
        const float Dm = Cm - cy, Nm = fmaf(Cm, cy, -1.0f);
        const float rm = rcp_fast(Dm);
        acc = fmaf(rm * rm, fmaf(twopi * (dx - 1.0f) * Sm, fmaf(-2.0f * Nm, rm, cy), Nm), acc);
    }
    // |k| = 2..4, first order, + side (E^-1) and - side (E)
    const float sp = fmaf(1.0f - twopi * dx, kA1, -twopi * kB1);
    const float sm = fmaf(1.0f + twopi * dx, kA1, -twopi * kB1);
    float far = 2.0f * cy * fmaf(Ei, sp, E * sm);
    // second order, k = 2
    {
        const float c2 = fmaf(2.0f * cy, cy, -1.0f), c4 = fmaf(-4.0f * cy, cy, 2.0f);
        const float tp = 2.0f * Ei * kQN2, tm = 2.0f * E * kQN2;
        far = fmaf(tp * tp, fmaf(twopi * (dx + 2.0f), c4, c2), far);
        far = fmaf(tm * tm, fmaf(twopi * (2.0f - dx), c4, c2), far);
    }
    return (acc + far) * kTwoPiSqF;
}

} // namespace sd
