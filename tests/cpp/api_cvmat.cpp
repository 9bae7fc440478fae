// The cv::Mat / CameraParams forms of the C++ drop-in headers, the signatures
// a reference caller uses (StereoSGBM::compute, StereoRectifier,
// rectifyImageGPU; include/stereo/sgbm_gpu.h:41 and rectification.h:49-97 of
// the reference).  Built by tests/test_cpp_api.py against a stand-in
// opencv2/core.hpp (tests/cpp/fake_opencv), since OpenCV's C++ headers are not
// installed here; with "gpu" it also checks every cv::Mat form against the
// raw-pointer form of the same call.
#include <cstdio>
#include <cstring>
#include <vector>

#include "stereo/rectification.h"
#include "stereo/sgbm_gpu.h"

#ifndef LUMEN_HAVE_OPENCV
#error "the cv::Mat forms are compiled only when <opencv2/core.hpp> is found"
#endif

#define CHECK(c)                                                       \
    do {                                                               \
        if (!(c)) {                                                    \
            std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c);  \
            return 1;                                                  \
        }                                                              \
    } while (0)

template <typename F>
static bool throws_stereo(F f) {
    try {
        f();
    } catch (const stereo::StereoException&) {
        return true;
    }
    return false;
}

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    const int W = 96, H = 64;
    stereo::CameraParams cp;
    cp.width = W;
    cp.height = H;
    cp.K0.create(3, 3, CV_64FC1);
    std::memset(cp.K0.data, 0, 9 * 8);
    cp.K0.at<double>(0, 0) = 1000.0;
    cp.K0.at<double>(1, 1) = 1200.0;
    cp.T.create(3, 1, CV_64FC1);
    cp.T.at<double>(0, 0) = 0.3;
    cp.T.at<double>(1, 0) = 0.0;
    cp.T.at<double>(2, 0) = 0.4;
    cp.computeDerivedValues();
    CHECK(cp.focalLength == 1100.0);
    CHECK(cp.baseline > 0.4999 && cp.baseline < 0.5001);

    // maps of the wrong type are rejected before anything touches the device
    stereo::CameraParams bad = cp;
    bad.map0x.create(H, W, CV_8UC1);
    bad.map0y.create(H, W, CV_32FC1);
    bad.map1x.create(H, W, CV_32FC1);
    bad.map1y.create(H, W, CV_32FC1);
    CHECK(throws_stereo([&] { stereo::StereoRectifier r(bad); }));

    // maps: a sub-pixel shift with some source points outside the image
    for (cv::Mat* m : {&cp.map0x, &cp.map0y, &cp.map1x, &cp.map1y}) m->create(H, W, CV_32FC1);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            cp.map0x.at<float>(y, x) = x * 1.01f - 0.7f;
            cp.map0y.at<float>(y, x) = y + 0.25f;
            cp.map1x.at<float>(y, x) = x + 0.5f;
            cp.map1y.at<float>(y, x) = y * 0.98f + 0.3f;
        }
    cv::Mat left(H, W, CV_8UC1), right(H, W, CV_8UC1);
    for (int i = 0; i < W * H; ++i) {
        left.data[i] = (uint8_t)(i * 37 + (i / W) * 11);
        right.data[i] = (uint8_t)(i * 53 + 7);
    }
    try {
        stereo::StereoRectifier rect(cp);
        CHECK(gpu);
        CHECK(!rect.isPreRectified());
        CHECK(rect.getParams().width == W);
        cv::Mat lr, rr;
        rect.rectify(left, right, lr, rr);
        CHECK(lr.rows == H && lr.cols == W && lr.type() == CV_8UC1 && rr.type() == CV_8UC1);
        std::vector<uint8_t> l2(W * H), r2(W * H);
        rect.rectify(left.data, right.data, 1, l2.data(), r2.data());
        CHECK(std::memcmp(lr.data, l2.data(), W * H) == 0);
        CHECK(std::memcmp(rr.data, r2.data(), W * H) == 0);
        // one image through the standalone function, gray and BGR
        cv::Mat one;
        stereo::rectifyImageGPU(left, cp.map0x, cp.map0y, one);
        CHECK(std::memcmp(one.data, l2.data(), W * H) == 0);
        cv::Mat bgr(H, W, CV_8UC3), bgrOut;
        for (int i = 0; i < W * H * 3; ++i) bgr.data[i] = (uint8_t)(i * 29 + 3);
        stereo::rectifyImageGPU(bgr, cp.map1x, cp.map1y, bgrOut);
        std::vector<uint8_t> b2(W * H * 3);
        stereo::rectifyImageGPU(bgr.data, cp.map1x.ptr<float>(), cp.map1y.ptr<float>(), b2.data(), W,
                                H, 3);
        CHECK(bgrOut.type() == CV_8UC3 && std::memcmp(bgrOut.data, b2.data(), b2.size()) == 0);
        // an image of another size than the calibration's
        cv::Mat small(H - 1, W, CV_8UC1);
        CHECK(throws_stereo([&] { rect.rectify(small, small, lr, rr); }));
        // pre-rectified: rectify clones
        stereo::CameraParams pre;
        pre.width = W;
        pre.height = H;
        stereo::StereoRectifier same(pre);
        CHECK(same.isPreRectified());
        same.rectify(left, right, lr, rr);
        CHECK(lr.data != left.data && std::memcmp(lr.data, left.data, W * H) == 0);
        // StereoSGBM::compute(cv::Mat...) equals the raw-pointer call
        stereo::StereoParams p;
        p.maxDisparity = 32;
        p.numDirections = 8;
        stereo::StereoSGBM sgbm(p);
        cv::Mat disp;
        sgbm.compute(left, right, disp);
        CHECK(disp.rows == H && disp.cols == W && disp.type() == CV_16SC1);
        std::vector<int16_t> d2(W * H);
        sgbm.compute(left.data, right.data, W, H, W, 1, d2.data(), W * 2);
        CHECK(std::memcmp(disp.data, d2.data(), W * H * 2) == 0);
        CHECK(throws_stereo([&] { sgbm.compute(left, small, disp); }));
        CHECK(throws_stereo([&] { sgbm.compute(cv::Mat(), right, disp); }));
    } catch (const stereo::CudaException& e) {
        CHECK(!gpu);
        CHECK(e.error_code == LUMEN_ERR_NO_DEVICE || e.error_code == LUMEN_ERR_CUDA);
    }
    std::printf("ok\n");
    return 0;
}
