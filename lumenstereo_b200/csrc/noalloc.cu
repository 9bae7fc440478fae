// noalloc.cu -- Census cost volume with no device allocation.
//
// lumen_census_cost_noalloc runs the two Census stages of the pipeline
// (census_kernel, census_cost_kernel in cost.cu) for callers that must not
// allocate device memory: code that enqueues work from a real-time loop where
// cudaMalloc's implicit device synchronisation would stall other streams, and
// plugin hosts that own every byte of device memory through their own pool.
// The caller passes the two gray images and the output volume; the only
// intermediate, the two Census descriptor images, lives in the file-scope
// array below.
//
// The array is part of the library's device image: every GPU that loads the
// library holds its 16 MiB until the process exits.  Every call shares it, so
// calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on it; serialise them.  Each call rewrites
// every descriptor it reads (border pixels get 0), so nothing has to be
// cleared between calls.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace lumen;

namespace {

// Largest image (pixels per view) the fixed scratch holds: 1920x1080 fits.
constexpr size_t kNoAllocMaxPixels = size_t(1) << 21;

// Census descriptors of the left view, then of the right view.
static __device__ __align__(256) uint32_t g_census_scratch[2 * kNoAllocMaxPixels];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Device address of g_census_scratch on the current device.  In host code the
// array's name is only a host-side stand-in for the symbol, never a device
// address, so the address is looked up once per device (with that device
// current) and cached.
lumen_status scratch_for_current_device(uint32_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return set_error(LUMEN_ERR_CUDA, std::string("lumen_census_cost_noalloc: cudaGetDevice: ") +
                                             cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT,
                         "lumen_census_cost_noalloc: device ordinal above 63 is not supported");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_census_scratch);
        if (e != cudaSuccess || !p)
            return set_error(LUMEN_ERR_CUDA,
                             std::string("lumen_census_cost_noalloc: cudaGetSymbolAddress: ") +
                                 cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return LUMEN_OK;
}

}  // namespace

extern "C" size_t lumen_census_cost_noalloc_max_pixels(void) { return kNoAllocMaxPixels; }

extern "C" lumen_status lumen_census_cost_noalloc(const uint8_t* d_left, const uint8_t* d_right,
                                                  int width, int height, int min_disparity,
                                                  int max_disparity, uint8_t* d_cost,
                                                  int cost_stride, void* stream) {
    if (!d_left || !d_right || !d_cost)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_census_cost_noalloc: NULL buffer");
    if (width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_census_cost_noalloc: empty image");
    const int D = max_disparity - min_disparity;
    if (min_disparity < 0 || D < 1)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT,
                         "lumen_census_cost_noalloc: need 0 <= minDisparity < maxDisparity");
    if (D > LUMEN_MAX_DISPARITY_RANGE)
        return set_error(LUMEN_ERR_RANGE_EXCEEDS_LIMIT,
                         "lumen_census_cost_noalloc: disparity range exceeds 512");
    // the same bound as the other entry points: keeps every index of the cost
    // kernel (x - minDisparity - d) inside int range
    if ((long long)max_disparity * 16 > 32767)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT,
                         "lumen_census_cost_noalloc: maxDisparity * 16 exceeds the int16 output range");
    // the cost kernel writes 16 disparities per 16-byte store
    if ((reinterpret_cast<uintptr_t>(d_cost) & 15u) != 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT,
                         "lumen_census_cost_noalloc: d_cost must be 16-byte aligned");
    if (cost_stride < D || cost_stride % 16 != 0 || cost_stride > 4096)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT,
                         "lumen_census_cost_noalloc: cost_stride must be a multiple of 16, "
                         ">= maxDisparity - minDisparity and <= 4096");
    if ((size_t)width * (size_t)height > kNoAllocMaxPixels)
        return set_error(LUMEN_ERR_OUT_OF_BUDGET,
                         "lumen_census_cost_noalloc: width*height = " +
                             std::to_string((size_t)width * (size_t)height) +
                             " exceeds the fixed scratch of " + std::to_string(kNoAllocMaxPixels) +
                             " pixels per view");
    uint32_t* scratch = nullptr;
    lumen_status st = scratch_for_current_device(&scratch);
    if (st != LUMEN_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t N = (size_t)width * height;
    launch_census(d_left, d_right, width, height, scratch, scratch + N, s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = launch_census_cost(scratch, scratch + N, width, height, D, cost_stride, min_disparity,
                               d_cost, s);
    if (e != cudaSuccess)
        return set_error(LUMEN_ERR_CUDA,
                         std::string("lumen_census_cost_noalloc: ") + cudaGetErrorString(e));
    return LUMEN_OK;
}
