// wave_inst.cuh -- launch helper of the schedule-4 wave kernel, instantiated
// once per padded disparity count (64 * KP) in wave_k<KP>.cu.
#pragma once
#include "wave_kernel.cuh"

namespace lumen {

// grid == 0: report the CTAs per SM that fit (occupancy) in *perSM, launch
// nothing.
template <int KW, bool WRAP, bool FULL, int NP, int R, int T = 32>
cudaError_t wave_launch_t(const WaveArgs& a, int smem, int grid, cudaStream_t s, int* perSM) {
    auto kern = wave_kernel<KW, WRAP, FULL, NP, R, T>;
    constexpr int threads = (R / (32 / T) + 2) * 32;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    if (grid == 0) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, kern, threads, smem);
    kern<<<grid, threads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int KW, int NP, int R, int T = 32>
cudaError_t wave_launch_np(const WaveArgs& a, bool wrap, bool full, int smem, int grid,
                           cudaStream_t s, int* perSM) {
    if (wrap) return full ? wave_launch_t<KW, true, true, NP, R, T>(a, smem, grid, s, perSM)
                          : wave_launch_t<KW, true, false, NP, R, T>(a, smem, grid, s, perSM);
    return full ? wave_launch_t<KW, false, true, NP, R, T>(a, smem, grid, s, perSM)
                : wave_launch_t<KW, false, false, NP, R, T>(a, smem, grid, s, perSM);
}

// Lane teams of T lanes (batched launches): words per lane KW = 64 * KP / (2 T).
template <int KP, int T>
cudaError_t wave_dispatch_team_kp(const WaveArgs& a, int R, int NP, bool wrap, bool full, int smem,
                                  int grid, cudaStream_t s, int* perSM) {
    constexpr int KW = 32 * KP / T;
    if (R == 8) return NP == 3 ? wave_launch_np<KW, 3, 8, T>(a, wrap, full, smem, grid, s, perSM)
                               : wave_launch_np<KW, 1, 8, T>(a, wrap, full, smem, grid, s, perSM);
    if (R == 16) return NP == 3 ? wave_launch_np<KW, 3, 16, T>(a, wrap, full, smem, grid, s, perSM)
                                : wave_launch_np<KW, 1, 16, T>(a, wrap, full, smem, grid, s, perSM);
    if (R == 32) return NP == 3 ? wave_launch_np<KW, 3, 32, T>(a, wrap, full, smem, grid, s, perSM)
                                : wave_launch_np<KW, 1, 32, T>(a, wrap, full, smem, grid, s, perSM);
    return cudaErrorInvalidValue;
}

template <int KP>
cudaError_t wave_dispatch_kp(const WaveArgs& a, int R, int NP, bool wrap, bool full, int smem,
                             int grid, cudaStream_t s, int* perSM) {
    constexpr int KW = KP;
    if (R == 4) return NP == 3 ? wave_launch_np<KW, 3, 4>(a, wrap, full, smem, grid, s, perSM)
                               : wave_launch_np<KW, 1, 4>(a, wrap, full, smem, grid, s, perSM);
    if (R == 8) return NP == 3 ? wave_launch_np<KW, 3, 8>(a, wrap, full, smem, grid, s, perSM)
                               : wave_launch_np<KW, 1, 8>(a, wrap, full, smem, grid, s, perSM);
    if (R == 16) return NP == 3 ? wave_launch_np<KW, 3, 16>(a, wrap, full, smem, grid, s, perSM)
                                : wave_launch_np<KW, 1, 16>(a, wrap, full, smem, grid, s, perSM);
    return cudaErrorInvalidValue;
}

}  // namespace lumen

#define LUMEN_WAVE_INSTANCE(KP)                                                                \
    namespace lumen {                                                                          \
    cudaError_t wave_dispatch_##KP(const WaveArgs& a, int R, int NP, bool wrap, bool full,     \
                                   int smem, int grid, cudaStream_t s, int* perSM) {           \
        return wave_dispatch_kp<KP>(a, R, NP, wrap, full, smem, grid, s, perSM);               \
    }                                                                                          \
    }

// team instances: 8 or 16 lanes for 64 and 128 padded disparities, 16 for 192 to 320
#define LUMEN_WAVE_TEAM_INSTANCE(KP, T)                                                        \
    namespace lumen {                                                                          \
    cudaError_t wave_dispatch_team_##KP##_##T(const WaveArgs& a, int R, int NP, bool wrap,     \
                                              bool full, int smem, int grid, cudaStream_t s,   \
                                              int* perSM) {                                    \
        return wave_dispatch_team_kp<KP, T>(a, R, NP, wrap, full, smem, grid, s, perSM);       \
    }                                                                                          \
    }
