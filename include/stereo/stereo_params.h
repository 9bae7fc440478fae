#pragma once
/**
 * stereo_params.h -- SGBM parameters, field for field as LumenStereo's
 * include/stereo/stereo_params.h:20-104 (same names, defaults and checks).
 */
#include "../lumen_sgbm.h"

#if defined(__has_include)
#if __has_include(<opencv2/core.hpp>)
#include <opencv2/core.hpp>
#define LUMEN_HAVE_OPENCV 1
#endif
#endif

namespace stereo {

enum class MatchingCostMode : int {
    SAD = 0,     // mean absolute difference over blockSize x blockSize (Sobel-x prefiltered)
    Census = 1,  // 5x5 census + Hamming distance
};

struct StereoParams {
    int minDisparity = 0;
    int maxDisparity = 128;
    int blockSize = 5;
    int P1 = 200;
    int P2 = 800;
    int preFilterCap = 31;
    int uniquenessRatio = 10;
    int disp12MaxDiff = 1;
    int speckleWindowSize = 100;
    int speckleRange = 32;
    bool useGPU = true;
    bool useSharedMemory = true;
    int numDirections = 4;
    MatchingCostMode matchingCostMode = MatchingCostMode::SAD;

    void autoComputePenalties(int numChannels = 1) {
        P1 = 8 * numChannels * blockSize * blockSize;
        P2 = 32 * numChannels * blockSize * blockSize;
    }

    bool isValid() const {
        if (blockSize < 1 || blockSize % 2 == 0) return false;
        if (minDisparity < 0) return false;
        if (maxDisparity <= minDisparity) return false;
        if (P2 <= P1) return false;
        if (uniquenessRatio < 0 || uniquenessRatio > 100) return false;
        return true;
    }

    lumen_stereo_params toC() const {
        lumen_stereo_params c;
        c.minDisparity = minDisparity;
        c.maxDisparity = maxDisparity;
        c.blockSize = blockSize;
        c.P1 = P1;
        c.P2 = P2;
        c.preFilterCap = preFilterCap;
        c.uniquenessRatio = uniquenessRatio;
        c.disp12MaxDiff = disp12MaxDiff;
        c.speckleWindowSize = speckleWindowSize;
        c.speckleRange = speckleRange;
        c.useGPU = useGPU ? 1 : 0;
        c.useSharedMemory = useSharedMemory ? 1 : 0;
        c.numDirections = numDirections;
        c.matchingCostMode = static_cast<int>(matchingCostMode);
        return c;
    }

    static StereoParams fromC(const lumen_stereo_params& c) {
        StereoParams p;
        p.minDisparity = c.minDisparity;
        p.maxDisparity = c.maxDisparity;
        p.blockSize = c.blockSize;
        p.P1 = c.P1;
        p.P2 = c.P2;
        p.preFilterCap = c.preFilterCap;
        p.uniquenessRatio = c.uniquenessRatio;
        p.disp12MaxDiff = c.disp12MaxDiff;
        p.speckleWindowSize = c.speckleWindowSize;
        p.speckleRange = c.speckleRange;
        p.useGPU = c.useGPU != 0;
        p.useSharedMemory = c.useSharedMemory != 0;
        p.numDirections = c.numDirections;
        p.matchingCostMode = static_cast<MatchingCostMode>(c.matchingCostMode);
        return p;
    }
};

#ifdef LUMEN_HAVE_OPENCV
/** Calibration of a camera pair, field for field as the reference's
 *  CameraParams (include/stereo/stereo_params.h:132-175).  The rectifier uses
 *  width, height and the four CV_32FC1 maps; empty maps mean the pair is
 *  already rectified. */
struct CameraParams {
    int width = 0;
    int height = 0;
    cv::Mat K0, D0;
    cv::Mat K1, D1;
    cv::Mat R, T;
    double baseline = 0.0;
    double focalLength = 0.0;
    int disparityOffset = 0;
    int numDisparities = 0;
    cv::Mat R0, R1;
    cv::Mat P0, P1;
    cv::Mat Q;
    cv::Mat map0x, map0y;
    cv::Mat map1x, map1y;

    /** baseline = |T|, focalLength = (fx + fy) / 2 of camera 0. */
    void computeDerivedValues() {
        if (!T.empty()) baseline = cv::norm(T);
        if (!K0.empty()) focalLength = (K0.at<double>(0, 0) + K0.at<double>(1, 1)) / 2.0;
    }
};
#endif

}  // namespace stereo
