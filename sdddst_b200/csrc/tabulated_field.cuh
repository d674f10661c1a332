// Tabulated periodic shear-stress field: the counterpart of the reference's
// PeriodicShearStressELTE (loadStress(pwd, "xy" | "xy_diff_x", 1024),
// python/src/periodic_shear_stress_ELTE_wrapper.cpp:40-46), whose C++ source
// and 1024 x 1024 data file are not part of the reference.  The tables are
// built here from the analytic periodic field (AnalyticField.cpp:145-181).
//
// The periodic field is singular only where a dislocation meets its own
// image-free term, tau_0 = dx (dx^2 - dy^2) / r^4 (the small-r limit of the
// y-periodic closed form); tau - tau_0 is smooth over the whole cell.  So a
// table holds the remainder R = tau - tau_0 (and R_x = tau_x - tau_0,x for
// the x-derivative) on a (G + 3) x (G + 3) grid of spacing 1/G covering
// [-0.5 - 1/G, 0.5 + 2/G]^2 (one guard point below, two above), and an
// evaluation is tau_0 in closed form plus a bicubic Catmull-Rom
// interpolation of R from the 4 x 4 neighbourhood (interpolation error
// O(G^-3) of R's third derivatives; the singular part stays exact).
//
// Shared by the device kernels and the host API (__host__ __device__).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace sd {

constexpr int kTabG = 1024;          // intervals per axis
constexpr int kTabS = kTabG + 3;     // stored points per axis

// grid coordinate of stored index k (k = 0 .. kTabS - 1)
__host__ __device__ inline double tab_coord(int k) { return -0.5 + (double)(k - 1) / (double)kTabG; }

// image-free edge dislocation field and its x-derivative
__host__ __device__ inline double tau0_xy(double dx, double dy)
{
    const double r2 = dx * dx + dy * dy;
    return dx * (dx * dx - dy * dy) / (r2 * r2);
}
__host__ __device__ inline double tau0_xy_dx(double dx, double dy)
{
    const double x2 = dx * dx, y2 = dy * dy, r2 = x2 + y2;
    return (-x2 * x2 + 6.0 * x2 * y2 - y2 * y2) / (r2 * r2 * r2);
}

__host__ __device__ inline void catmull_rom(double t, double w[4])
{
    const double t2 = t * t, t3 = t2 * t;
    w[0] = 0.5 * (-t3 + 2.0 * t2 - t);
    w[1] = 0.5 * (3.0 * t3 - 5.0 * t2 + 2.0);
    w[2] = 0.5 * (-3.0 * t3 + 4.0 * t2 + t);
    w[3] = 0.5 * (t3 - t2);
}

// bicubic interpolation of a remainder table at (dx, dy) in [-0.5, 0.5]^2
__host__ __device__ inline double tab_interp(const double *tab, double dx, double dy)
{
    const double u = (dx + 0.5) * kTabG, v = (dy + 0.5) * kTabG;
    int ix = (int)floor(u), iy = (int)floor(v);
    ix = ix < 0 ? 0 : (ix > kTabG - 1 ? kTabG - 1 : ix);
    iy = iy < 0 ? 0 : (iy > kTabG - 1 ? kTabG - 1 : iy);
    double wx[4], wy[4];
    catmull_rom(u - ix, wx);
    catmull_rom(v - iy, wy);
    double acc = 0.0;
    for (int b = 0; b < 4; ++b) {
        // stored index of grid point ix + a - 1 is ix + a (one guard point)
        const double *row = tab + (long)(iy + b) * kTabS + ix;
        const double s = wx[0] * row[0] + wx[1] * row[1] + wx[2] * row[2] + wx[3] * row[3];
        acc += wy[b] * s;
    }
    return acc;
}

} // namespace sd
