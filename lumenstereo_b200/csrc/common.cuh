// common.cuh -- shared definitions of the B200 SGBM kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace lumen {

constexpr int kMaxD = 512;      // stereo::kSgbmMaxDisparityRange (include/stereo/sgbm_limits.h:9)
constexpr int kWarp = 32;
constexpr unsigned kFullMask = 0xFFFFFFFFu;

// Disparities per volume row are padded to a multiple of 64 (two per 16-bit
// lane pair, 32 lanes): every warp lane owns 2*KW consecutive disparities,
// i.e. KW packed uint16x2 words, and the padded bytes of the uint8 cost volume
// are 0 so they never influence a minimum.
inline int padded_d(int D) { return ((D + 63) / 64) * 64; }
inline int words_per_lane(int D) { return padded_d(D) / 64; }

// Parameters of the SGM recurrence shared by every aggregation kernel.
struct SgmConsts {
    int W, H, D, Dp;
    int P1, P2;
    int costScale;
    // derived
    uint32_t p1x2;     // P1 (mod 2^16) in both halves
    uint32_t bsub;     // boundary stand-in (0xFFFF - P1) in both halves (no-wrap mode)
};

// Everything a kernel needs to know about one stereo pair's volumes.
struct PairView {
    const uint8_t* cost;    // [H][W][Dp] uint8
    const uint8_t* img;     // [H][W] left gray image (adaptive P2 input)
    uint16_t* agg;          // [H][W][Dp] uint16
};

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
    return __byte_perm(a, b, s);
}

// bytes (b0,b1,b2,b3) of a word -> two uint16x2 words (b0,b1) and (b2,b3)
__device__ __forceinline__ uint32_t bytes_lo(uint32_t v) { return __byte_perm(v, 0u, 0x4140); }
__device__ __forceinline__ uint32_t bytes_hi(uint32_t v) { return __byte_perm(v, 0u, 0x4342); }

}  // namespace lumen
