// depth.cu -- the two stages on either side of the disparity map.
//
// lumen_disparity_to_depth_device replaces disparityToDepthGPU /
// disparityToDepthKernel (src/depth_map.cu:74-102, 169-187): depth =
// f * B / (d / 16 + doffs) for positive 1/16-px disparities, 0 otherwise,
// with the reference's expression order.  Compiled with --use_fast_math like
// the reference, so the division is the same approximate one.
//
// lumen_rectify_maps_device generates the CV_32FC1 rectification maps on the
// device from a camera's intrinsics, distortion, rectifying rotation and new
// projection (the maps the reference gets from cv::initUndistortRectifyMap,
// src/calibration.cpp:253-266), so a served calibration needs no host
// OpenCV.  The model is the published pinhole camera with Brown-Conrady
// distortion (k1, k2, p1, p2, k3): for every rectified pixel (u, v) the ray
// (P'R)^-1 (u, v, 1) is projected to (x, y), distorted by
//   r2 = x^2 + y^2,  s = 1 + k1 r2 + k2 r2^2 + k3 r2^3,
//   xd = x s + 2 p1 x y + p2 (r2 + 2 x^2),  yd = y s + p1 (r2 + 2 y^2) + 2 p2 x y,
// and mapped through K: map = (fx xd + cx, fy yd + cy).  Computed in double
// and stored as float.
#include <cmath>
#include <string>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

__global__ void __launch_bounds__(256)
depth_kernel(const int16_t* __restrict__ disp, size_t dispPitch, int W, int H, float focal,
             float baseline, float doffs, float* __restrict__ depth, size_t depthPitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const int16_t d = disp[(size_t)y * dispPitch + x];
    float z = 0.0f;
    if (d > 0) {
        const float dispFloat = static_cast<float>(d) / 16.0f;
        const float denom = dispFloat + doffs;
        z = (denom > 0.0f) ? ((focal * baseline) / denom) : 0.0f;
    }
    depth[(size_t)y * depthPitch + x] = z;
}

struct MapParams {
    double iR[9];        // (P[:, :3] R)^-1
    double fx, fy, cx, cy;
    double k1, k2, p1, p2, k3;
};

__global__ void __launch_bounds__(256)
rectify_map_kernel(MapParams m, int W, int H, float* __restrict__ mapX, float* __restrict__ mapY) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    if (u >= W) return;
    const double X = m.iR[0] * u + m.iR[1] * v + m.iR[2];
    const double Y = m.iR[3] * u + m.iR[4] * v + m.iR[5];
    const double Z = m.iR[6] * u + m.iR[7] * v + m.iR[8];
    const double w = Z != 0.0 ? 1.0 / Z : 1.0;
    const double x = X * w, y = Y * w;
    const double x2 = x * x, y2 = y * y, r2 = x2 + y2, xy2 = 2.0 * x * y;
    const double s = 1.0 + ((m.k3 * r2 + m.k2) * r2 + m.k1) * r2;
    const double xd = x * s + m.p1 * xy2 + m.p2 * (r2 + 2.0 * x2);
    const double yd = y * s + m.p1 * (r2 + 2.0 * y2) + m.p2 * xy2;
    mapX[(size_t)v * W + u] = (float)(m.fx * xd + m.cx);
    mapY[(size_t)v * W + u] = (float)(m.fy * yd + m.cy);
}

static bool invert3(const double a[9], double r[9]) {
    const double c0 = a[4] * a[8] - a[5] * a[7];
    const double c1 = a[5] * a[6] - a[3] * a[8];
    const double c2 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c0 + a[1] * c1 + a[2] * c2;
    if (det == 0.0 || !std::isfinite(det)) return false;
    const double id = 1.0 / det;
    r[0] = c0 * id;
    r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    r[3] = c1 * id;
    r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    r[6] = c2 * id;
    r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

}  // namespace lumen

using namespace lumen;

extern "C" lumen_status lumen_disparity_to_depth_device(const int16_t* d_disp, int width, int height,
                                                        size_t disp_stride, float focal_px,
                                                        float baseline, float disparity_offset_px,
                                                        float* d_depth, size_t depth_stride,
                                                        void* stream) {
    if (!d_disp || !d_depth || width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_disparity_to_depth_device: empty input");
    if (!disp_stride) disp_stride = (size_t)width * 2;
    if (!depth_stride) depth_stride = (size_t)width * 4;
    if (disp_stride < (size_t)width * 2 || disp_stride % 2 || depth_stride < (size_t)width * 4 || depth_stride % 4)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_disparity_to_depth_device: bad stride");
    dim3 g((width + 255) / 256, height);
    depth_kernel<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_disp, disp_stride / 2, width, height,
                                                                   focal_px, baseline, disparity_offset_px,
                                                                   d_depth, depth_stride / 4);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(LUMEN_ERR_CUDA, std::string("lumen_disparity_to_depth_device: ") + cudaGetErrorString(e));
    return LUMEN_OK;
}

extern "C" lumen_status lumen_rectify_maps_device(const double K[9], const double dist[5], const double R[9],
                                                  const double P[12], int width, int height, float* d_map_x,
                                                  float* d_map_y, void* stream) {
    if (!K || !R || !P || !d_map_x || !d_map_y || width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_rectify_maps_device: NULL or empty argument");
    // P[:, :3] * R, row-major 3x4 P
    double PR[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            PR[3 * i + j] = P[4 * i + 0] * R[0 + j] + P[4 * i + 1] * R[3 + j] + P[4 * i + 2] * R[6 + j];
    MapParams m{};
    if (!invert3(PR, m.iR))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_rectify_maps_device: singular P*R");
    m.fx = K[0];
    m.fy = K[4];
    m.cx = K[2];
    m.cy = K[5];
    if (dist) {
        m.k1 = dist[0];
        m.k2 = dist[1];
        m.p1 = dist[2];
        m.p2 = dist[3];
        m.k3 = dist[4];
    }
    dim3 g((width + 255) / 256, height);
    rectify_map_kernel<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(m, width, height, d_map_x, d_map_y);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(LUMEN_ERR_CUDA, std::string("lumen_rectify_maps_device: ") + cudaGetErrorString(e));
    return LUMEN_OK;
}
