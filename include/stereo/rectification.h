#pragma once
/**
 * rectification.h -- drop-in for LumenStereo's stereo::StereoRectifier and
 * rectifyImageGPU (include/stereo/rectification.h:41-97), over the C ABI.
 * Maps are CV_32FC1 (width*height floats); without maps the pair is
 * pre-rectified and rectify() copies.
 */
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "../lumen_sgbm.h"
#include "common.h"

namespace stereo {

class StereoRectifier {
public:
    StereoRectifier(int width, int height, const float* map0x = nullptr,
                    const float* map0y = nullptr, const float* map1x = nullptr,
                    const float* map1y = nullptr) {
        throwOnError(lumen_rectifier_create(width, height, map0x, map0y, map1x, map1y, &r_));
    }
    ~StereoRectifier() { lumen_rectifier_destroy(r_); }
    StereoRectifier(const StereoRectifier&) = delete;
    StereoRectifier& operator=(const StereoRectifier&) = delete;

    bool isPreRectified() const { return lumen_rectifier_is_pre_rectified(r_) != 0; }

    void rectify(const uint8_t* leftRaw, const uint8_t* rightRaw, int channels, uint8_t* leftRect,
                 uint8_t* rightRect) {
        throwOnError(lumen_rectifier_rectify(r_, leftRaw, rightRaw, channels, leftRect, rightRect));
    }

private:
    lumen_rectifier* r_ = nullptr;
};

inline void rectifyImageGPU(const uint8_t* src, const float* mapX, const float* mapY, uint8_t* dst,
                            int width, int height, int channels) {
    throwOnError(lumen_remap(src, mapX, mapY, dst, width, height, channels));
}

}  // namespace stereo
