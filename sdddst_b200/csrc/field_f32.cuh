// FP32 field kernels of the mixed-precision path: tau_xy for the pair sum
// (two pairs at a time, packed) and d tau_xy / dx for the Jacobian.
//
// Same image structure as field_f64.cuh (AnalyticField.cpp:145-160).  The
// caller forms the separation in FP64 (so close pairs keep full relative
// accuracy) and rounds it to FP32 once; the image terms run in FP32 with the
// SFU (ex2, rcp).
//  * sin(pi dy), |dy| <= 0.5: an odd degree-13 polynomial (Taylor; the
//    remainder is below 7e-10) in the Jacobian; the pair sum takes it from
//    its caller, formed in FP64 as sin(pi y_i) cos(pi y_j) - cos(pi y_i)
//    sin(pi y_j) (only its square enters, so the image in y is immaterial);
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

// ---------------------------------------------------------------------------
// tau_xy of two pairs at once in packed FP32 (sm_100 FFMA2 / FMUL2 / FADD2:
// one issue slot per two lanes' arithmetic; the SFU work stays scalar),
// arranged so that one pair needs two ex2 and one rcp:
//  * sh = sinh(pi dx) from its odd series below |pi dx| = 0.5, else from
//    e^{+-pi dx}; with E = e^{2 pi dx}:  E + 1/E = sigma = 2 + 4 sh^2 and
//    (E - 1/E) / 2 = dl = sinh(2 pi dx) = sh (e^{pi dx} + e^{-pi dx}),
//    E^2 + E^-2 = sigma^2 - 2, E^2 - E^-2 = 2 sigma dl;
//  * C_{+-1} = cosh(2 pi (dx +- 1)) = (E e^{+-2 pi} + E^-1 e^{-+2 pi}) / 2, a
//    sum of two positive terms (the sigma/dl form cancels near |dx| = 1/2);
//  * the k = 0 and |k| = 1 terms over one common denominator
//    s^2 D+^2 D-^2 (s = sh^2 + sin^2(pi dy), D+- = C+- - cos(2 pi dy)),
//    whose factors lie in [1e-26, 1e17] for separations above 1e-7.
// dx is the minimum-image separation, sn = sin(pi dy).  Returns
// 2 tau_xy / (2 pi^2), so the caller's factor is pi^2; s is handed back for
// the close-pair prefilter (s <= pi^2 r^2 (1 + pi^2 r^2 / 2)).
__device__ __forceinline__ float2 f2c(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float ex2_fast(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

constexpr float kPiLog2eF = 4.532360141827193f;   // pi log2(e)
constexpr float kSinhSplitF = 0.15915494309189535f; // |pi dx| = 0.5
constexpr float kPiSqF = 9.869604401089358f;

__device__ __forceinline__ float2 tau_xy_f32x2(float2 dx, float2 sn, float2 &s_out)
{
    const float2 sn2 = mul2(sn, sn);
    const float2 cy = fma2(sn2, f2c(-2.0f), f2c(1.0f));
    // sinh(pi dx): series in dx (coefficients pi^{2k+1} / (2k+1)!) or exponentials
    const float2 x2 = mul2(dx, dx);
    float2 q = fma2(x2, f2c(0.5992645293207919f), f2c(2.550164039877345f));
    q = fma2(q, x2, f2c(5.167712780049969f));
    q = fma2(q, x2, f2c(3.141592653589793f));
    q = mul2(dx, q);
    const float2 xk = mul2(dx, f2c(kPiLog2eF));
    float2 ep, epi;
    ep.x = ex2_fast(xk.x);
    ep.y = ex2_fast(xk.y);
    epi.x = ex2_fast(-xk.x);
    epi.y = ex2_fast(-xk.y);
    const float2 shx = fma2(ep, f2c(0.5f), mul2(epi, f2c(-0.5f)));
    float2 sh;
    sh.x = fabsf(dx.x) < kSinhSplitF ? q.x : shx.x;
    sh.y = fabsf(dx.y) < kSinhSplitF ? q.y : shx.y;
    const float2 sh2 = mul2(sh, sh);
    const float2 s = add2(sh2, sn2);
    s_out = s;
    const float2 n0 = fma2(sn2, f2c(-1.0f), mul2(sh2, cy)); // sh^2 cy - sn^2
    const float2 dl = mul2(sh, add2(ep, epi));               // sinh(2 pi dx)
    const float2 sg = fma2(sh2, f2c(4.0f), f2c(2.0f));       // E + 1/E
    const float2 E = mul2(ep, ep), Ei = mul2(epi, epi);
    const float2 cp = fma2(E, f2c(0.5f * kQP1), mul2(Ei, f2c(0.5f * kQN1)));
    const float2 cm = fma2(E, f2c(0.5f * kQN1), mul2(Ei, f2c(0.5f * kQP1)));
    const float2 dp = fma2(cy, f2c(-1.0f), cp), dm = fma2(cy, f2c(-1.0f), cm);
    const float2 np = fma2(cp, cy, f2c(-1.0f)), nm = fma2(cm, cy, f2c(-1.0f));
    const float2 dp2 = mul2(dp, dp), dm2 = mul2(dm, dm);
    const float2 s2 = mul2(s, s), pq = mul2(dp2, dm2);
    const float2 den = mul2(s2, pq);
    float2 r;
    r.x = rcp_fast(den.x);
    r.y = rcp_fast(den.y);
    // 2 [dx n0 / (2 s^2) + (dx + 1) N+ / D+^2 + (dx - 1) N- / D-^2]
    const float2 u = mul2(fma2(dx, f2c(2.0f), f2c(2.0f)), np);
    const float2 w = mul2(fma2(dx, f2c(2.0f), f2c(-2.0f)), nm);
    const float2 bs = fma2(u, dm2, mul2(w, dp2));
    const float2 near2 = mul2(fma2(mul2(dx, n0), pq, mul2(s2, bs)), r);
    // 2 x the |k| >= 2 first-order sums and the k = 2 second order
    const float2 g1 = fma2(dx, mul2(sg, f2c(4.0f * kA1)), mul2(dl, f2c(-8.0f * kB1)));
    const float2 g2 = fma2(dx, fma2(sg, sg, f2c(-2.0f)), mul2(mul2(sg, dl), f2c(-4.0f)));
    const float2 c2 = fma2(mul2(cy, cy), f2c(16.0f * kQN2SQ), f2c(-8.0f * kQN2SQ));
    const float2 far2 = fma2(c2, g2, mul2(cy, g1));
    return add2(near2, far2);
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

// tau_xy_dx_f32 for two pairs at once in packed FP32 (same terms and the same
// order of operations as the scalar form; the SFU calls stay scalar).
__device__ __forceinline__ float2 tau_xy_dx_f32x2(float2 dx, float2 dy)
{
    const float twopi = 6.28318530717959f;
    const float2 y2 = mul2(dy, dy);
    float2 p = fma2(f2c(0.00046630280576761f), y2, f2c(-0.00737043094571435f));
    p = fma2(p, y2, f2c(0.08214588661112823f));
    p = fma2(p, y2, f2c(-0.59926452932079207f));
    p = fma2(p, y2, f2c(2.55016403987734549f));
    p = fma2(p, y2, f2c(-5.16771278004997003f));
    p = fma2(p, y2, f2c(3.14159265358979324f));
    const float2 sn = mul2(dy, p);
    const float2 sn2 = mul2(sn, sn);
    const float2 cy = fma2(f2c(-2.0f), sn2, f2c(1.0f));
    const float2 a = mul2(f2c(kPiF), dx);
    float2 ep, epi;
    ep.x = __expf(a.x);
    ep.y = __expf(a.y);
    epi.x = __expf(-a.x);
    epi.y = __expf(-a.y);
    const float2 a2 = mul2(a, a);
    const float2 poly =
        mul2(a, fma2(a2, fma2(a2, fma2(a2, f2c(1.0f / 5040.0f), f2c(1.0f / 120.0f)), f2c(1.0f / 6.0f)), f2c(1.0f)));
    const float2 shx = mul2(f2c(0.5f), fma2(epi, f2c(-1.0f), ep));
    float2 sh;
    sh.x = fabsf(a.x) < 0.5f ? poly.x : shx.x;
    sh.y = fabsf(a.y) < 0.5f ? poly.y : shx.y;
    const float2 ch = mul2(f2c(0.5f), add2(ep, epi));
    const float2 sh2 = mul2(sh, sh);
    const float2 E = mul2(ep, ep), Ei = mul2(epi, epi);
    // k = 0
    const float2 D0 = mul2(f2c(2.0f), add2(sh2, sn2));
    const float2 N0 = fma2(mul2(f2c(-4.0f), sh2), sn2, mul2(f2c(2.0f), fma2(sn2, f2c(-1.0f), sh2)));
    const float2 S0 = mul2(mul2(f2c(2.0f), sh), ch);
    float2 r0;
    r0.x = rcp_fast(D0.x);
    r0.y = rcp_fast(D0.y);
    float2 acc = mul2(mul2(r0, r0), fma2(mul2(mul2(f2c(twopi), dx), S0), fma2(mul2(f2c(-2.0f), N0), r0, cy), N0));
    // |k| = 1
    {
        const float2 ap = mul2(E, f2c(kQP1)), bp = mul2(Ei, f2c(kQN1));
        const float2 Cp = mul2(f2c(0.5f), add2(ap, bp)), Sp = mul2(f2c(0.5f), fma2(bp, f2c(-1.0f), ap));
        const float2 Dp = fma2(cy, f2c(-1.0f), Cp), Np = fma2(Cp, cy, f2c(-1.0f));
        float2 rp;
        rp.x = rcp_fast(Dp.x);
        rp.y = rcp_fast(Dp.y);
        acc = fma2(mul2(rp, rp),
                   fma2(mul2(mul2(f2c(twopi), add2(dx, f2c(1.0f))), Sp), fma2(mul2(f2c(-2.0f), Np), rp, cy), Np),
                   acc);
        const float2 am = mul2(E, f2c(kQN1)), bm = mul2(Ei, f2c(kQP1));
        const float2 Cm = mul2(f2c(0.5f), add2(am, bm)), Sm = mul2(f2c(0.5f), fma2(bm, f2c(-1.0f), am));
        const float2 Dm = fma2(cy, f2c(-1.0f), Cm), Nm = fma2(Cm, cy, f2c(-1.0f));
        float2 rm;
        rm.x = rcp_fast(Dm.x);
        rm.y = rcp_fast(Dm.y);
        acc = fma2(mul2(rm, rm),
                   fma2(mul2(mul2(f2c(twopi), add2(dx, f2c(-1.0f))), Sm), fma2(mul2(f2c(-2.0f), Nm), rm, cy), Nm),
                   acc);
    }
    // |k| = 2..4, first order, + side (E^-1) and - side (E)
    const float2 sp = fma2(fma2(f2c(-twopi), dx, f2c(1.0f)), f2c(kA1), f2c(-twopi * kB1));
    const float2 sm = fma2(fma2(f2c(twopi), dx, f2c(1.0f)), f2c(kA1), f2c(-twopi * kB1));
    float2 far = mul2(mul2(f2c(2.0f), cy), fma2(Ei, sp, mul2(E, sm)));
    // second order, k = 2
    {
        const float2 c2 = fma2(mul2(f2c(2.0f), cy), cy, f2c(-1.0f)), c4 = fma2(mul2(f2c(-4.0f), cy), cy, f2c(2.0f));
        const float2 tp = mul2(mul2(f2c(2.0f), Ei), f2c(kQN2)), tm = mul2(mul2(f2c(2.0f), E), f2c(kQN2));
        far = fma2(mul2(tp, tp), fma2(mul2(f2c(twopi), add2(dx, f2c(2.0f))), c4, c2), far);
        far = fma2(mul2(tm, tm), fma2(mul2(f2c(twopi), fma2(dx, f2c(-1.0f), f2c(2.0f))), c4, c2), far);
    }
    return mul2(add2(acc, far), f2c(kTwoPiSqF));
}

} // namespace sd
