// Allocation-free velocity evaluation.
//
// sdddst_speeds() and every context need device memory from cudaMalloc.  Some
// callers cannot allocate: a host application whose stepping loop runs inside
// a device-memory budget owned by another framework, or code that issues work
// between other kernels on a stream, where cudaMalloc's implicit device-wide
// synchronisation would stall everything else.  For them the O(N^2) pair sum
// has one variant whose scratch (the per-tile partial sums) lives in a
// statically sized __device__ array of this library instead of in allocated
// memory.  The caller passes the inputs and the output in device memory.
#include "engine.h"

#include <mutex>

namespace sd {
namespace {

constexpr int kNoAllocMaxN = 4096; // largest N this entry point accepts
constexpr int kNoAllocTile = 64;   // pair-sum tile for N < 8192 (pair_tile_size)
constexpr int kNoAllocBlocks = kNoAllocMaxN / kNoAllocTile;
// 64 x 4096 doubles = 2 MiB; every GPU that loads the library holds it until exit.
constexpr size_t kNoAllocDoubles = (size_t)kNoAllocBlocks * kNoAllocMaxN;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch[kMaxDevices] = {nullptr};

} // namespace
} // namespace sd

static __device__ __align__(256) double sdddst_noalloc_scratch[sd::kNoAllocDoubles];

extern "C" int sdddst_speeds_noalloc(int n, const double *x_device, const double *y_device, const double *b_device,
                                     double tau_ext, double *v_device, void *stream)
{
    using namespace sd;
    if (n < 2 || n > kNoAllocMaxN) return SDDDST_ERR_CAPACITY; // N above the static scratch's size
    if (!x_device || !y_device || !b_device || !v_device) return SDDDST_ERR_INVALID;
    if (pair_part_doubles(n) > kNoAllocDoubles) return SDDDST_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SDDDST_ERR_CUDA;
    double *scratch;
    {
        // The array's host-side name is not a device address: look the address
        // up once per device, with that device current.
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch[dev]) {
            void *ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, sdddst_noalloc_scratch) != cudaSuccess || !ptr) return SDDDST_ERR_CUDA;
            g_scratch[dev] = static_cast<double *>(ptr);
        }
        scratch = g_scratch[dev];
    }
    launch_speeds_raw(n, x_device, y_device, b_device, tau_ext, scratch, v_device, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? SDDDST_OK : SDDDST_ERR_CUDA;
}
