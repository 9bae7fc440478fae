#pragma once
/**
 * point_cloud.h -- drop-in for LumenStereo's point cloud and PLY export
 * (include/stereo/point_cloud.h:17-62), header-only: the back-projection runs
 * on the device through the C ABI (lumen_depth_to_points), the PLY writers are
 * host code writing the same files as exportPLY / exportPLY_ASCII
 * (src/point_cloud.cpp:57-127).
 */
#include <cstddef>
#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

#include "../lumen_sgbm.h"
#include "common.h"

#if defined(__has_include)
#if __has_include(<opencv2/core.hpp>)
#include <opencv2/core.hpp>
#define LUMEN_HAVE_OPENCV 1
#endif
#endif

namespace stereo {

struct Point3D {
    float x, y, z;
    uint8_t r, g, b;

    Point3D() : x(0), y(0), z(0), r(255), g(255), b(255) {}
    Point3D(float x_, float y_, float z_) : x(x_), y(y_), z(z_), r(255), g(255), b(255) {}
    Point3D(float x_, float y_, float z_, uint8_t r_, uint8_t g_, uint8_t b_)
        : x(x_), y(y_), z(z_), r(r_), g(g_), b(b_) {}
};

/** Pixels with 0 < Z <= 100 as points ((u - cx) Z / fx, (v - cy) Z / fy, Z) in
 *  raster order, coloured from `bgr` (3 bytes a pixel, NULL: white).  Host
 *  buffers; strides in bytes (0: packed). */
inline std::vector<Point3D> depthToPointCloud(const float* depth, int width, int height, size_t depthStride,
                                              const uint8_t* bgr, size_t bgrStride, double fx, double fy,
                                              double cx, double cy) {
    std::vector<lumen_point3d> raw((size_t)width * height);
    int n = 0;
    throwOnError(lumen_depth_to_points(depth, width, height, depthStride, bgr, bgrStride, fx, fy, cx, cy,
                                       raw.data(), &n));
    std::vector<Point3D> points;
    points.reserve(n);
    for (int i = 0; i < n; ++i)
        points.emplace_back(raw[i].x, raw[i].y, raw[i].z, raw[i].r, raw[i].g, raw[i].b);
    return points;
}

#ifdef LUMEN_HAVE_OPENCV
/** depth CV_32FC1; color CV_8UC3 (used when its size matches); K0 the 3x3
 *  CV_64F intrinsics of the reference's CameraParams. */
inline std::vector<Point3D> depthToPointCloud(const cv::Mat& depth, const cv::Mat& color, const cv::Mat& K0) {
    if (depth.empty() || depth.type() != CV_32FC1) throw StereoException("depth must be CV_32FC1");
    const bool hasColor = !color.empty() && color.size() == depth.size() && color.type() == CV_8UC3;
    return depthToPointCloud(depth.ptr<float>(), depth.cols, depth.rows, depth.step, hasColor ? color.data : nullptr,
                             hasColor ? color.step : 0, K0.at<double>(0, 0), K0.at<double>(1, 1),
                             K0.at<double>(0, 2), K0.at<double>(1, 2));
}
#endif

inline void writePlyHeader(std::ostream& f, const char* format, size_t n) {
    f << "ply\nformat " << format << " 1.0\nelement vertex " << n
      << "\nproperty float x\nproperty float y\nproperty float z\n"
         "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n";
}

inline bool exportPLY_ASCII(const std::vector<Point3D>& points, const std::string& filename) {
    std::ofstream f(filename);
    if (!f.is_open()) return false;
    writePlyHeader(f, "ascii", points.size());
    for (const Point3D& p : points)
        f << p.x << ' ' << p.y << ' ' << p.z << ' ' << int(p.r) << ' ' << int(p.g) << ' ' << int(p.b) << '\n';
    return true;
}

/** binary: little-endian x, y, z float32 then r, g, b (15 bytes a point). */
inline bool exportPLY(const std::vector<Point3D>& points, const std::string& filename, bool binary = true) {
    if (!binary) return exportPLY_ASCII(points, filename);
    std::ofstream f(filename, std::ios::binary);
    if (!f.is_open()) return false;
    writePlyHeader(f, "binary_little_endian", points.size());
    std::vector<char> rec(points.size() * 15);
    char* o = rec.data();
    for (const Point3D& p : points) {
        const float xyz[3] = {p.x, p.y, p.z};
        for (int k = 0; k < 12; ++k) o[k] = reinterpret_cast<const char*>(xyz)[k];   // host is little-endian
        o[12] = char(p.r);
        o[13] = char(p.g);
        o[14] = char(p.b);
        o += 15;
    }
    f.write(rec.data(), (std::streamsize)rec.size());
    return true;
}

}  // namespace stereo
