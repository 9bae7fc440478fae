// dpx_probe.cu -- issue rate of the packed uint16x2 operations the SGM
// recurrence can be written with (lumen_debug_op_rates).
//
// The recurrence step (sgm_step.cuh, wave_kernel.cuh) takes, per packed word,
// two minima and an add before the final add-subtract.  It can be written
// with two-input minima (__vminu2) and plain adds, or with the three-input
// forms sm_90+ offers (__vimin3_u16x2: min of three; __viaddmin_u16x2:
// min(a + b, c)).  Which is cheaper depends on their issue rate, which this
// probe measures: each kernel runs 16 independent chains per thread of one
// operation over 2048 steps on every SM (8 CTAs of 8 warps per SM), timed
// with CUDA events; the result is device time per warp-instruction per SM.
#include <cuda_runtime.h>

#include <string>

#include "../../include/lumen_sgbm.h"
#include "kernels.cuh"

namespace lumen {

constexpr int kProbeChains = 16;
constexpr int kProbeSteps = 2048;

// OP 0: __vminu2; 1: __vimin3_u16x2; 2: __viaddmin_u16x2; 3: 32-bit add
template <int OP>
__global__ void __launch_bounds__(256) op_rate_kernel(uint32_t seed, uint32_t* sink) {
    uint32_t v[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) v[c] = seed * (threadIdx.x + 1) + c * 0x9E3779B9u;
    const uint32_t k1 = seed ^ 0x00120034u, k2 = seed ^ 0x56007800u;
    for (int s = 0; s < kProbeSteps; ++s) {
        // step operands with no closed form over the loop (one pair per step,
        // shared by the 16 chains)
        const uint32_t x = k1 ^ ((uint32_t)s * 0x01000193u), y = k2 ^ ((uint32_t)s * 0x9E3779B1u);
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) {
            if (OP == 0) v[c] = __vminu2(v[c], x);
            if (OP == 1) v[c] = __vimin3_u16x2(v[c], x, y);
            if (OP == 2) v[c] = __viaddmin_u16x2(v[c], x, y);
            if (OP == 3) v[c] = v[c] + x;
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) acc ^= v[c];
    if (acc == 0x12345678u) sink[threadIdx.x] = acc;  // keeps the chains live
}

}  // namespace lumen

using namespace lumen;

// ns per warp-instruction per SM of each operation (out[0..3]: __vminu2,
// __vimin3_u16x2, __viaddmin_u16x2, 32-bit add); the loop's own counter and
// operand work is spread over the 16 chains and included in every figure alike.
extern "C" lumen_status lumen_debug_op_rates(float* out4) {
    if (!out4) return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_debug_op_rates: NULL output");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set_error(LUMEN_ERR_NO_DEVICE, "lumen_debug_op_rates: no CUDA device");
    uint32_t* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&sink, 256 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int blocks = sms * 8;
    for (int op = 0; op < 4 && e == cudaSuccess; ++op) {
        auto launch = [&]() {
            switch (op) {
            case 0: op_rate_kernel<0><<<blocks, 256>>>(7u, sink); break;
            case 1: op_rate_kernel<1><<<blocks, 256>>>(7u, sink); break;
            case 2: op_rate_kernel<2><<<blocks, 256>>>(7u, sink); break;
            default: op_rate_kernel<3><<<blocks, 256>>>(7u, sink); break;
            }
        };
        launch();  // warm-up
        e = cudaEventRecord(a);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) launch();
        if (e == cudaSuccess) e = cudaEventRecord(b);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        const double warpInstrPerSM = 5.0 * 8 * 8 * (double)kProbeChains * kProbeSteps;
        out4[op] = (float)(ms * 1e6 / warpInstrPerSM);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (sink) cudaFree(sink);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (e != cudaSuccess) return set_error(LUMEN_ERR_CUDA, std::string("lumen_debug_op_rates: ") + cudaGetErrorString(e));
    return LUMEN_OK;
}
