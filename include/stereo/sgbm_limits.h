#pragma once
/**
 * sgbm_limits.h -- disparity-range limit of the B200 SGBM engine.
 * Same names and values as LumenStereo's include/stereo/sgbm_limits.h:9-22.
 */
#include "../lumen_sgbm.h"

namespace stereo {

inline constexpr int kSgbmMaxDisparityRange = LUMEN_MAX_DISPARITY_RANGE;  // 512

/** Middlebury ndisp clamped to the engine limit (fallback when missing). */
inline int middleburyMatcherMaxDisparity(int calibNumDisparities, int fallbackWhenMissing = 96) {
    const int ndisp = (calibNumDisparities > 0) ? calibNumDisparities : fallbackWhenMissing;
    return (ndisp > kSgbmMaxDisparityRange) ? kSgbmMaxDisparityRange : ndisp;
}

}  // namespace stereo
