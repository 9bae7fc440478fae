#pragma once
/**
 * sgbm_gpu.h -- drop-in replacement for LumenStereo's stereo::StereoSGBM
 * (include/stereo/sgbm_gpu.h:29-91), header-only over the C ABI in
 * include/lumen_sgbm.h.  Link with liblumen_sgbm.so.
 *
 *   stereo::StereoSGBM sgbm(params);
 *   sgbm.compute(leftRect, rightRect, disparity);   // cv::Mat overload when OpenCV is present
 *   sgbm.compute(l, r, w, h, stride, channels, out, out_stride);  // raw pointers
 */
#include <cstddef>
#include <cstdint>

#include "../lumen_sgbm.h"
#include "common.h"
#include "sgbm_limits.h"
#include "stereo_params.h"  // defines LUMEN_HAVE_OPENCV when OpenCV headers exist

namespace stereo {

class StereoSGBM {
public:
    explicit StereoSGBM(const StereoParams& params = StereoParams()) : params_(params) {
        const lumen_stereo_params c = params_.toC();
        throwOnError(lumen_sgbm_create(&c, &h_));
    }
    ~StereoSGBM() { lumen_sgbm_destroy(h_); }
    StereoSGBM(const StereoSGBM&) = delete;
    StereoSGBM& operator=(const StereoSGBM&) = delete;

    /** Host buffers: gray (channels 1) or BGR (3) rows of width*channels bytes
     *  with pitch `stride`; out: int16 disparities in 1/16 px (-1 invalid). */
    void compute(const uint8_t* left, const uint8_t* right, int width, int height, size_t stride,
                 int channels, int16_t* out, size_t outStride) {
        throwOnError(lumen_sgbm_compute(h_, left, right, width, height, stride, channels, out,
                                        outStride));
    }

    /** Device buffers on a CUDA stream (cudaStream_t as void*), asynchronous. */
    void computeDevice(const uint8_t* dLeft, const uint8_t* dRight, int width, int height,
                       size_t stride, int channels, int16_t* dOut, size_t outStride,
                       void* stream = nullptr) {
        throwOnError(lumen_sgbm_compute_device(h_, dLeft, dRight, width, height, stride, channels,
                                               dOut, outStride, stream));
    }

#ifdef LUMEN_HAVE_OPENCV
    /** src/sgbm_gpu.cu:147-195: CV_8UC1 or CV_8UC3 (BGR) in, CV_16SC1 out. */
    void compute(const cv::Mat& left, const cv::Mat& right, cv::Mat& disparity) {
        if (left.empty() || right.empty()) throw StereoException("Input images are empty");
        if (left.size() != right.size())
            throw StereoException("Left and right images must have same size");
        if (left.channels() != right.channels())
            throw StereoException("Left and right images must have the same channel count");
        cv::Mat l = left.isContinuous() ? left : left.clone();
        cv::Mat r = right.isContinuous() ? right : right.clone();
        disparity.create(left.rows, left.cols, CV_16SC1);
        compute(l.data, r.data, l.cols, l.rows, l.step[0], l.channels(),
                reinterpret_cast<int16_t*>(disparity.data), disparity.step[0]);
    }
#endif

    void setParams(const StereoParams& params) {
        params_ = params;
        const lumen_stereo_params c = params_.toC();
        throwOnError(lumen_sgbm_set_params(h_, &c));
    }
    const StereoParams& getParams() const { return params_; }

    float getLastComputeTimeMs() const { return timing(0); }
    float getCostComputeTimeMs() const { return timing(1); }
    float getAggregationTimeMs() const { return timing(2); }
    float getPostProcessTimeMs() const { return timing(3); }

private:
    float timing(int i) const {
        float t[4] = {0, 0, 0, 0};
        throwOnError(lumen_sgbm_get_timings(h_, t));
        return t[i];
    }
    StereoParams params_;
    lumen_sgbm* h_ = nullptr;
};

}  // namespace stereo
