#pragma once
/**
 * depth_map.h -- drop-in for LumenStereo's GPU depth functions
 * (include/stereo/depth_map.h:33-56), header-only over the C ABI in
 * include/lumen_sgbm.h, with device pointers where the reference takes
 * CudaBuffer.  Asynchronous on `stream` (cudaStream_t as void*, NULL: the
 * default stream); errors throw like the rest of the API.
 */
#include <cstddef>
#include <cstdint>

#include "../lumen_sgbm.h"
#include "common.h"

namespace stereo {

/** depth = f * B / (d / 16 + doffs) for positive 1/16-px disparities, 0
 *  elsewhere; packed width x height buffers. */
inline void disparityToDepthGPU(const int16_t* dDisparity, float* dDepth, int width, int height,
                                float focalLength, float baseline, float disparityOffsetPx = 0.0f,
                                void* stream = nullptr) {
    throwOnError(lumen_disparity_to_depth_device(dDisparity, width, height, 0, focalLength, baseline,
                                                 disparityOffsetPx, dDepth, 0, stream));
}

/** Colour index 0 where z <= 0 or z > 2 maxDepth, else
 *  (int)((1 - clamp((z - minDepth) / (maxDepth - minDepth), 0, 1)) * 255), looked
 *  up in `lut` (host, 256 triplets in output order); 3 bytes a pixel. */
inline void colorizeDepthGPU(const float* dDepth, uint8_t* dColorized, int width, int height,
                             float minDepth, float maxDepth, const uint8_t* lut, void* stream = nullptr) {
    throwOnError(lumen_depth_colorize_device(dDepth, width, height, 0, minDepth, maxDepth, lut, dColorized, 0,
                                             stream));
}

/** Both in one pass over the disparity map (dDepth may be NULL). */
inline void disparityToDepthColorGPU(const int16_t* dDisparity, float* dDepth, uint8_t* dColorized, int width,
                                     int height, float focalLength, float baseline, float disparityOffsetPx,
                                     float minDepth, float maxDepth, const uint8_t* lut,
                                     void* stream = nullptr) {
    throwOnError(lumen_disparity_to_depth_color_device(dDisparity, width, height, 0, focalLength, baseline,
                                                       disparityOffsetPx, dDepth, 0, minDepth, maxDepth, lut,
                                                       dColorized, 0, stream));
}

}  // namespace stereo
