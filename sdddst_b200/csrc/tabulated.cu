// Builds the remainder tables of the tabulated field (tabulated_field.cuh)
// from the FP64 analytic periodic field: R = tau - tau_0 and
// R_x = tau_x - tau_0,x at every stored grid point.  At the origin, where
// tau and tau_0 are both singular, R takes its limit by Richardson
// extrapolation of symmetric four-point averages (error O(delta^4)).
#include "engine.h"
#include "field_f64.cuh"
#include "tabulated_field.cuh"

namespace sd {

namespace {

__device__ double rem_xy(double x, double y) { return tau_xy_f64(x, y) - tau0_xy(x, y); }
__device__ double rem_dx(double x, double y) { return tau_xy_dx_f64(x, y) - tau0_xy_dx(x, y); }

template <bool kDx>
__device__ double rem_at_origin()
{
    auto avg = [](double d) {
        double s;
        if (kDx) s = rem_dx(d, 0.0) + rem_dx(-d, 0.0) + rem_dx(0.0, d) + rem_dx(0.0, -d);
        else s = rem_xy(d, 0.0) + rem_xy(-d, 0.0) + rem_xy(0.0, d) + rem_xy(0.0, -d);
        return 0.25 * s;
    };
    const double d = 2e-3;
    return (4.0 * avg(0.5 * d) - avg(d)) / 3.0;
}

__global__ void tab_build_kernel(double *__restrict__ txy, double *__restrict__ tdx)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)kTabS * kTabS) return;
    const int kx = (int)(idx % kTabS), ky = (int)(idx / kTabS);
    const double x = tab_coord(kx), y = tab_coord(ky);
    if (x == 0.0 && y == 0.0) {
        txy[idx] = rem_at_origin<false>();
        tdx[idx] = rem_at_origin<true>();
    } else {
        txy[idx] = rem_xy(x, y);
        tdx[idx] = rem_dx(x, y);
    }
}

} // namespace

int tabulated_build(Engine &e)
{
    const size_t count = (size_t)kTabS * kTabS;
    if (!e.d_tab_xy && (cudaMalloc(&e.d_tab_xy, sizeof(double) * count) != cudaSuccess ||
                        cudaMalloc(&e.d_tab_dx, sizeof(double) * count) != cudaSuccess)) {
        e.err = "tabulated field: out of device memory";
        return SDDDST_ERR_NOMEM;
    }
    tab_build_kernel<<<(unsigned)((count + 255) / 256), 256, 0, e.st>>>(e.d_tab_xy, e.d_tab_dx);
    e.launches++;
    return e.sync_check("tabulated field");
}

} // namespace sd
