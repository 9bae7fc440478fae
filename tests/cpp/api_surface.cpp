// Compiles against the C++ drop-in headers and exercises the parts of the API
// that need no GPU (parameters, limits, error mapping).  Built and run by
// tests/test_cpp_api.py.
#include <cstdio>
#include <cstring>

#include "stereo/rectification.h"
#include "stereo/sgbm_gpu.h"

#define CHECK(c)                                                       \
    do {                                                               \
        if (!(c)) {                                                    \
            std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c);  \
            return 1;                                                  \
        }                                                              \
    } while (0)

int main(int argc, char** argv) {
    stereo::StereoParams p;
    CHECK(p.minDisparity == 0 && p.maxDisparity == 128 && p.blockSize == 5);
    CHECK(p.isValid());
    p.blockSize = 4;
    CHECK(!p.isValid());
    p.blockSize = 5;
    p.autoComputePenalties(1);
    CHECK(p.P1 == 200 && p.P2 == 800);
    CHECK(stereo::kSgbmMaxDisparityRange == 512);
    CHECK(stereo::middleburyMatcherMaxDisparity(600) == 512);
    lumen_stereo_params c;
    lumen_stereo_params_default(&c);
    CHECK(std::memcmp(&c, &(const lumen_stereo_params&)stereo::StereoParams().toC(), sizeof c) == 0);
    CHECK(stereo::StereoParams::fromC(c).numDirections == 4);
    bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    try {
        stereo::StereoSGBM sgbm(p);
        CHECK(gpu);  // construction succeeds only with a device
        uint8_t img[64 * 64] = {0};
        int16_t out[64 * 64];
        bool threw = false;
        try {
            stereo::StereoParams big;
            big.maxDisparity = stereo::kSgbmMaxDisparityRange + 32;
            sgbm.setParams(big);
            sgbm.compute(img, img, 64, 64, 64, 1, out, 128);
        } catch (const stereo::StereoException&) {
            threw = true;
        }
        CHECK(threw);
        sgbm.setParams(p);
        sgbm.compute(img, img, 64, 64, 64, 1, out, 128);
        CHECK(sgbm.getLastComputeTimeMs() > 0.f);
    } catch (const stereo::CudaException& e) {
        CHECK(!gpu);
        CHECK(e.error_code == LUMEN_ERR_NO_DEVICE);
    }
    std::printf("ok\n");
    return 0;
}
