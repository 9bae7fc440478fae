// Compiles against the C++ drop-in headers and exercises the parts of the API
// that need no GPU (parameters, limits, error mapping).  Built and run by
// tests/test_cpp_api.py.
#include <cstdio>
#include <cstring>

#include <fstream>
#include <sstream>

#include "stereo/depth_map.h"
#include "stereo/point_cloud.h"
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
    // PLY writers: the header and a 15-byte record per point / one text line
    std::vector<stereo::Point3D> pts = {stereo::Point3D(0.1f, -2.5f, 3.f, 255, 1, 200), stereo::Point3D(1.f, 2.f, 1e-7f)};
    const char* bin = "_api_surface_test.ply";
    CHECK(stereo::exportPLY(pts, bin));
    {
        std::ifstream f(bin, std::ios::binary);
        std::stringstream ss;
        ss << f.rdbuf();
        const std::string s = ss.str();
        const std::string head = "ply\nformat binary_little_endian 1.0\nelement vertex 2\n";
        CHECK(s.compare(0, head.size(), head) == 0);
        const size_t at = s.find("end_header\n") + 11;
        CHECK(s.size() == at + 30);
        float x;
        std::memcpy(&x, s.data() + at, 4);
        CHECK(x == 0.1f && (uint8_t)s[at + 12] == 255 && (uint8_t)s[at + 14] == 200 && (uint8_t)s[at + 29] == 255);
    }
    CHECK(stereo::exportPLY(pts, bin, false));
    {
        std::ifstream f(bin);
        std::stringstream ss;
        ss << f.rdbuf();
        const std::string s = ss.str();
        CHECK(s.substr(s.find("end_header\n") + 11) == "0.1 -2.5 3 255 1 200\n1 2 1e-07 255 255 255\n");
    }
    std::remove(bin);
    CHECK(!stereo::exportPLY(pts, "no_such_dir/x.ply"));
    // device-free argument checks of the depth entry points
    bool threwArg = false;
    try {
        stereo::disparityToDepthGPU(nullptr, nullptr, 4, 4, 1.f, 1.f);
    } catch (const stereo::StereoException&) {
        threwArg = true;
    }
    CHECK(threwArg);
    float depth[6] = {1.f, 0.f, 2.f, 200.f, -1.f, 3.f};
    uint8_t bgr[18];
    for (int i = 0; i < 18; ++i) bgr[i] = (uint8_t)i;
    try {
        std::vector<stereo::Point3D> cloud = stereo::depthToPointCloud(depth, 3, 2, 0, bgr, 0, 100.0, 100.0, 1.0, 0.5);
        CHECK(gpu);
        CHECK(cloud.size() == 3);
        CHECK(cloud[0].z == 1.f && cloud[0].r == 2 && cloud[0].b == 0);
        CHECK(cloud[1].z == 2.f && cloud[1].x == (float)((2 - 1.0) * 2.0 / 100.0));
        CHECK(cloud[2].z == 3.f && cloud[2].y == (float)((1 - 0.5) * 3.0 / 100.0) && cloud[2].r == 17);
    } catch (const stereo::CudaException& e) {
        CHECK(!gpu);
        CHECK(e.error_code == LUMEN_ERR_NO_DEVICE);
    }
    std::printf("ok\n");
    return 0;
}
