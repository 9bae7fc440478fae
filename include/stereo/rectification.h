#pragma once
/**
 * rectification.h -- drop-in for LumenStereo's stereo::StereoRectifier and
 * rectifyImageGPU (include/stereo/rectification.h:41-97), over the C ABI.
 *
 * With OpenCV headers present the reference's own signatures compile
 * unchanged: StereoRectifier(const CameraParams&), rectify(const cv::Mat&,
 * const cv::Mat&, cv::Mat&, cv::Mat&), getParams(), and
 * rectifyImageGPU(const cv::Mat&, const cv::Mat&, const cv::Mat&, cv::Mat&).
 * The raw-pointer forms are always there.  Maps are CV_32FC1 (width*height
 * floats); without maps the pair is pre-rectified and rectify() copies.
 */
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "../lumen_sgbm.h"
#include "common.h"
#include "stereo_params.h"  // CameraParams and LUMEN_HAVE_OPENCV when OpenCV headers exist

namespace stereo {

class StereoRectifier {
public:
    StereoRectifier(int width, int height, const float* map0x = nullptr,
                    const float* map0y = nullptr, const float* map1x = nullptr,
                    const float* map1y = nullptr) {
        throwOnError(lumen_rectifier_create(width, height, map0x, map0y, map1x, map1y, &r_));
    }
#ifdef LUMEN_HAVE_OPENCV
    /** src/rectification.cu:259-284: the maps are uploaded once; empty maps
     *  mean the pair is pre-rectified. */
    explicit StereoRectifier(const CameraParams& params) : params_(params) {
        const bool pre = params.map0x.empty() || params.map0y.empty();
        if (!pre) {
            checkMap(params.map0x, params);
            checkMap(params.map0y, params);
            checkMap(params.map1x, params);
            checkMap(params.map1y, params);
        }
        throwOnError(lumen_rectifier_create(
            params.width, params.height, pre ? nullptr : params.map0x.ptr<float>(),
            pre ? nullptr : params.map0y.ptr<float>(), pre ? nullptr : params.map1x.ptr<float>(),
            pre ? nullptr : params.map1y.ptr<float>(), &r_));
    }
#endif
    ~StereoRectifier() { lumen_rectifier_destroy(r_); }
    StereoRectifier(const StereoRectifier&) = delete;
    StereoRectifier& operator=(const StereoRectifier&) = delete;

    bool isPreRectified() const { return lumen_rectifier_is_pre_rectified(r_) != 0; }

    void rectify(const uint8_t* leftRaw, const uint8_t* rightRaw, int channels, uint8_t* leftRect,
                 uint8_t* rightRect) {
        throwOnError(lumen_rectifier_rectify(r_, leftRaw, rightRaw, channels, leftRect, rightRect));
    }

#ifdef LUMEN_HAVE_OPENCV
    /** src/rectification.cu:286-345: pre-rectified pairs are cloned; else both
     *  images are remapped into freshly created outputs of the input type.
     *  The images must have the calibration's size (the reference reads its
     *  maps past their end otherwise; here it is a StereoException). */
    void rectify(const cv::Mat& leftRaw, const cv::Mat& rightRaw, cv::Mat& leftRect,
                 cv::Mat& rightRect) {
        if (isPreRectified()) {
            leftRect = leftRaw.clone();
            rightRect = rightRaw.clone();
            return;
        }
        if (leftRaw.empty() || rightRaw.empty()) throw StereoException("Input images are empty");
        if (leftRaw.cols != params_.width || leftRaw.rows != params_.height ||
            rightRaw.cols != params_.width || rightRaw.rows != params_.height)
            throw StereoException("image size differs from the calibration's");
        if (leftRaw.type() != rightRaw.type())
            throw StereoException("Left and right images must have the same type");
        const cv::Mat l = leftRaw.isContinuous() ? leftRaw : leftRaw.clone();
        const cv::Mat r = rightRaw.isContinuous() ? rightRaw : rightRaw.clone();
        leftRect.create(l.rows, l.cols, l.type());
        rightRect.create(r.rows, r.cols, r.type());
        rectify(l.data, r.data, l.channels(), leftRect.data, rightRect.data);
    }

    const CameraParams& getParams() const { return params_; }
#endif

private:
#ifdef LUMEN_HAVE_OPENCV
    static void checkMap(const cv::Mat& m, const CameraParams& p) {
        if (m.type() != CV_32FC1 || m.cols != p.width || m.rows != p.height || !m.isContinuous())
            throw StereoException("rectification maps must be contiguous CV_32FC1 of the image size");
    }
    CameraParams params_;
#endif
    lumen_rectifier* r_ = nullptr;
};

inline void rectifyImageGPU(const uint8_t* src, const float* mapX, const float* mapY, uint8_t* dst,
                            int width, int height, int channels) {
    throwOnError(lumen_remap(src, mapX, mapY, dst, width, height, channels));
}

#ifdef LUMEN_HAVE_OPENCV
/** src/rectification.cu:354-411: one image; dst is created with src's type. */
inline void rectifyImageGPU(const cv::Mat& src, const cv::Mat& mapX, const cv::Mat& mapY,
                            cv::Mat& dst) {
    if (src.empty()) throw StereoException("Input image is empty");
    if (mapX.type() != CV_32FC1 || mapY.type() != CV_32FC1 || mapX.cols != src.cols ||
        mapX.rows != src.rows || mapY.cols != src.cols || mapY.rows != src.rows)
        throw StereoException("rectification maps must be CV_32FC1 of the image size");
    const cv::Mat s = src.isContinuous() ? src : src.clone();
    const cv::Mat mx = mapX.isContinuous() ? mapX : mapX.clone();
    const cv::Mat my = mapY.isContinuous() ? mapY : mapY.clone();
    dst.create(s.rows, s.cols, s.type());
    rectifyImageGPU(s.data, mx.ptr<float>(), my.ptr<float>(), dst.data, s.cols, s.rows,
                    s.channels());
}
#endif

}  // namespace stereo
