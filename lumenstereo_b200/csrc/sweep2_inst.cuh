// sweep2_inst.cuh -- launch helper of the schedule-3 sweep kernel, instantiated
// once per words-per-lane count KW in sweep2_k<KW>.cu.
#pragma once
#include "sweep2_kernel.cuh"

namespace lumen {

// grid == 0: report the CTAs per SM that fit (occupancy) in *perSM, launch nothing.
template <int KW, bool WRAP, bool FULL, int NP, int R>
cudaError_t sweep2_launch_t(const Sweep2Args& a, int smem, int grid, cudaStream_t s, int* perSM) {
    auto kern = sweep2_kernel<KW, WRAP, FULL, NP, R>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    if (grid == 0) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, kern, (R + 2) * 32, smem);
    kern<<<grid, (R + 2) * 32, smem, s>>>(a);
    return cudaGetLastError();
}

template <int KW, int NP, int R>
cudaError_t sweep2_launch_np(const Sweep2Args& a, bool wrap, bool full, int smem, int grid,
                             cudaStream_t s, int* perSM) {
    if (wrap) return full ? sweep2_launch_t<KW, true, true, NP, R>(a, smem, grid, s, perSM)
                          : sweep2_launch_t<KW, true, false, NP, R>(a, smem, grid, s, perSM);
    return full ? sweep2_launch_t<KW, false, true, NP, R>(a, smem, grid, s, perSM)
                : sweep2_launch_t<KW, false, false, NP, R>(a, smem, grid, s, perSM);
}

template <int KW>
cudaError_t sweep2_dispatch_kw(const Sweep2Args& a, int R, int NP, bool wrap, int smem, int grid,
                               cudaStream_t s, int* perSM) {
    const bool full = (a.D == a.Dp);
    if (R == 4) return NP == 3 ? sweep2_launch_np<KW, 3, 4>(a, wrap, full, smem, grid, s, perSM)
                               : sweep2_launch_np<KW, 1, 4>(a, wrap, full, smem, grid, s, perSM);
    if (R == 8) return NP == 3 ? sweep2_launch_np<KW, 3, 8>(a, wrap, full, smem, grid, s, perSM)
                               : sweep2_launch_np<KW, 1, 8>(a, wrap, full, smem, grid, s, perSM);
    return cudaErrorInvalidValue;
}

}  // namespace lumen

#define LUMEN_SWEEP2_INSTANCE(KW)                                                              \
    namespace lumen {                                                                          \
    cudaError_t sweep2_dispatch_##KW(const Sweep2Args& a, int R, int NP, bool wrap, int smem,  \
                                     int grid, cudaStream_t s, int* perSM) {                   \
        return sweep2_dispatch_kw<KW>(a, R, NP, wrap, smem, grid, s, perSM);                   \
    }                                                                                          \
    }
