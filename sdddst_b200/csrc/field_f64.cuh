// FP64 field kernels of the periodic edge-dislocation stress
// (reference: Fields/AnalyticField.cpp:24-181, ANALYTIC_FIELD_N = 4).
//
// The reference evaluates, per pair, ten y-periodic image columns
// f(u) = 2 pi^2 u (cosh 2pi u cos 2pi dy - 1)/(cosh 2pi u - cos 2pi dy)^2 at
// u = dx + k, each with its own cosh(), weighted by 1 for |k| <= 4 except the
// edge image (+4 for dx >= 0, -4 for dx < 0) weighted 1-|dx| and an end image
// (-5 resp. +5) weighted |dx|.  Here one expm1(pi dx) gives E = e^{2 pi dx},
// and every image's cosh/sinh is E q^k / 2 +- 1/(2 E q^k) with the constants
// q^k = e^{2 pi k}.  The k = 0 column uses the exact identities
//   cosh 2a - cos 2b = 2 (sinh^2 a + sin^2 b),
//   cosh 2a cos 2b - 1 = 2 (sinh^2 a - sin^2 b) - 4 sinh^2 a sin^2 b,
// (a = pi dx, b = pi dy) which stay accurate as r -> 0, where the reference
// switches to a 6th-order Taylor branch (r^2 <= 1e-6).  All image
// denominators are inverted with one division (prefix-product inversion).
#pragma once

#include "common.cuh"

namespace sd {

// In-place reciprocals of a[0..M-1] with one division: prefix products,
// invert the total, then peel off each factor.
template <int M>
__device__ __forceinline__ void batch_rcp(double (&a)[M])
{
    double pre[M];
    pre[0] = a[0];
#pragma unroll
    for (int k = 1; k < M; ++k) pre[k] = pre[k - 1] * a[k];
    double inv = 1.0 / pre[M - 1];
#pragma unroll
    for (int k = M - 1; k >= 1; --k) {
        double ak = a[k];
        a[k] = inv * pre[k - 1];
        inv = inv * ak;
    }
    a[0] = inv;
}

// Image table of one separation: u, N = C cy - 1, D = C - cy, S = sinh(2 pi u)
// and the weight w for the ten images in the order
//   [0] k=0, [1..4] k=+1..+4, [5..8] k=-1..-4, [9] end image (-5 or +5).
struct Images {
    double u[10], N[10], D[10], S[10], w[10];
    double cy;
    bool pos;
};

template <bool kNeedS>
__device__ __forceinline__ void make_images(double dx, double dy, Images &im)
{
    double sn = sinpi(dy);
    double sn2 = sn * sn;
    double cy = 1.0 - 2.0 * sn2; // cos(2 pi dy)
    double em1 = expm1(kPi * dx);
    double ep = 1.0 + em1;       // e^{pi dx}
    double E = ep * ep;          // e^{2 pi dx}
    double Ei = 1.0 / E;
    double sh = 0.5 * (em1 + em1 * ep * Ei); // sinh(pi dx)
    double sh2 = sh * sh;
    im.cy = cy;
    im.pos = dx >= 0.0;
    im.u[0] = dx;
    im.D[0] = 2.0 * (sh2 + sn2);
    im.N[0] = 2.0 * (sh2 - sn2) - 4.0 * sh2 * sn2;
    im.w[0] = 1.0;
    if (kNeedS) {
        double ch = 0.5 * (ep + ep * Ei); // cosh(pi dx)
        im.S[0] = 2.0 * sh * ch;
    }
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        double a = E * qpos(k), b = Ei * qneg(k); // e^{2pi(dx+k)}, e^{-2pi(dx+k)}
        double C = 0.5 * (a + b);
        im.u[k] = dx + (double)k;
        im.N[k] = C * cy - 1.0;
        im.D[k] = C - cy;
        if (kNeedS) im.S[k] = 0.5 * (a - b);
        double c = E * qneg(k), d = Ei * qpos(k); // e^{2pi(dx-k)}, e^{-2pi(dx-k)}
        double Cm = 0.5 * (c + d);
        im.u[4 + k] = dx - (double)k;
        im.N[4 + k] = Cm * cy - 1.0;
        im.D[4 + k] = Cm - cy;
        if (kNeedS) im.S[4 + k] = 0.5 * (c - d);
        im.w[k] = 1.0;
        im.w[4 + k] = 1.0;
    }
    // edge images and end image
    im.w[4] = im.pos ? 1.0 - dx : 1.0;
    im.w[8] = im.pos ? 1.0 : 1.0 + dx;
    {
        double a = im.pos ? E * qneg(5) : E * qpos(5);
        double b = im.pos ? Ei * qpos(5) : Ei * qneg(5);
        double C = 0.5 * (a + b);
        im.u[9] = im.pos ? dx - 5.0 : dx + 5.0;
        im.N[9] = C * cy - 1.0;
        im.D[9] = C - cy;
        if (kNeedS) im.S[9] = 0.5 * (a - b);
        im.w[9] = fabs(dx);
    }
}

// AnalyticField::xy (AnalyticField.cpp:145-160).
__device__ __forceinline__ double tau_xy_f64(double dx, double dy)
{
    Images im;
    make_images<false>(dx, dy, im);
    double inv[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) inv[k] = im.D[k] * im.D[k];
    batch_rcp<10>(inv);
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 10; ++k) acc += im.w[k] * im.u[k] * im.N[k] * inv[k];
    return acc * kTwoPiSq;
}

// AnalyticField::xy_diff_x (AnalyticField.cpp:162-181): d tau_xy / d dx,
//   sum_k w_k f'(u_k) + sigma (f(u_end) - f(u_edge)),  sigma = sign(dx),
//   f'(u) = 2 pi^2 / D^2 [N + 2 pi u S (cy - 2 N / D)].
__device__ __forceinline__ double tau_xy_dx_f64(double dx, double dy)
{
    Images im;
    make_images<true>(dx, dy, im);
    double inv[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) inv[k] = im.D[k];
    batch_rcp<10>(inv);
    const double twopi = 2.0 * kPi;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        double i2 = inv[k] * inv[k];
        double fp = i2 * (im.N[k] + twopi * im.u[k] * im.S[k] * (im.cy - 2.0 * im.N[k] * inv[k]));
        acc += im.w[k] * fp;
    }
    int edge = im.pos ? 4 : 8;
    double f_end = im.u[9] * im.N[9] * inv[9] * inv[9];
    double f_edge = im.u[edge] * im.N[edge] * inv[edge] * inv[edge];
    acc += im.pos ? (f_end - f_edge) : (f_edge - f_end);
    return acc * kTwoPiSq;
}

// AnalyticField::xy_diff_x2 (AnalyticField.cpp:95-132,183-202), the value
// the reference's eigenvalue derivatives use:
//   sum_k w_k F(u_k) + 2 sigma (f'(u_end) - f'(u_edge)),  sigma = sign(dx),
// where the reference's per-image term f_dx2 carries no 2 pi^2 factor (its f
// and f_dx do), so F = f'' / (2 pi^2):
//   F(u) = 4 pi / D^2 [S (cy - 2N/D) + pi u ((C - 2 S^2/D)(cy - 2N/D) - 2 (S^2/D)(cy - N/D))]
// with C = cosh 2 pi u = D + cy.
__device__ __forceinline__ double tau_xy_dx2_f64(double dx, double dy)
{
    Images im;
    make_images<true>(dx, dy, im);
    double inv[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) inv[k] = im.D[k];
    batch_rcp<10>(inv);
    const double twopi = 2.0 * kPi;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        const double r = inv[k], S = im.S[k], N = im.N[k], cy = im.cy;
        const double C = im.D[k] + cy, s2r = S * S * r, a = cy - 2.0 * N * r;
        const double F = 4.0 * kPi * r * r * (S * a + kPi * im.u[k] * ((C - 2.0 * s2r) * a - 2.0 * s2r * (cy - N * r)));
        acc += im.w[k] * F;
    }
    const int edge = im.pos ? 4 : 8;
    auto fprime = [&](int k) {
        const double r = inv[k];
        return kTwoPiSq * r * r * (im.N[k] + twopi * im.u[k] * im.S[k] * (im.cy - 2.0 * im.N[k] * r));
    };
    const double d = fprime(9) - fprime(edge);
    acc += im.pos ? 2.0 * d : -2.0 * d;
    return acc;
}

// Point-defect force term of calculateSpeeds (simulation.cpp:111-128):
// returns 2 A X(dx) X(dy) ((1-e)/s - K e)/s (subtracted times b_i) and the
// tolerance distance s = X2(dx) + X2(dy), with X, X2 as in utility.h:42-50.
__device__ __forceinline__ double pd_force_f64(double dx, double dy, double A, double K, double *s_out)
{
    double sx, cx, sy, cyy;
    sincospi(2.0 * dx, &sx, &cx);
    sincospi(2.0 * dy, &sy, &cyy);
    double Xx = sx * 0.5 / kPi, Xy = sy * 0.5 / kPi;
    double x2 = (1.0 - cx) * 0.5 / kPi / kPi;
    double y2 = (1.0 - cyy) * 0.5 / kPi / kPi;
    double s = x2 + y2;
    double e = exp(-K * s);
    *s_out = s;
    return 2.0 * A * Xx * Xy * ((1. - e) / s - K * e) / s;
}

// d/dx of the point-defect force divided by b (the diagonal seed of
// calculateJacobian, simulation.cpp:274-325), kept in the reference's three
// terms:  -A cx sy phi/(pi s) - A sx sy (e K sx/(pi s) - (1-e) sx/(pi s^2)
// + K^2 e sx/pi)/(2 pi^2 s) + A sx^2 sy phi/(2 pi^3 s^2), phi = (1-e)/s - K e.
__device__ __forceinline__ double pd_force_dx_f64(double dx, double dy, double A, double K)
{
    double sx, cx, sy, cyy;
    sincospi(2.0 * dx, &sx, &cx);
    sincospi(2.0 * dy, &sy, &cyy);
    const double ipi2 = 1.0 / (kPi * kPi);
    double s = (1.0 - cx) * ipi2 / 2.0 + (1.0 - cyy) * ipi2 / 2.0;
    double e = exp(-K * s);
    double phi = (1.0 - e) / s - K * e;
    double t1 = -A * cx / kPi * sy * phi / s;
    double t2 = -A * sx * ipi2 * sy * (e * K * sx / kPi / s - (1.0 - e) / (s * s) * sx / kPi + K * K * e * sx / kPi) / s / 2.0;
    double t3 = A * sx * sx * (ipi2 / kPi) * sy * phi / (s * s) / 2.0;
    return t1 + t2 + t3;
}

} // namespace sd
