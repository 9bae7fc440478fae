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
//
// lumen_depth_colorize_device replaces colorizeDepthKernel (src/depth_map.cu:
// 104-142): the colour index of a depth z is 0 for z <= 0 or z > 2 max, else
// (int)((1 - clamp((z - min) / (max - min), 0, 1)) * 255), looked up in a
// caller-given 256-entry table of channel triplets.  Fused with the depth
// conversion (lumen_disparity_to_depth_device with an RGB output) the pair
// runs as one pass over the disparity map: 2 B read and 4 + 3 B written per
// pixel, where the reference's two kernels re-read the depth map.
//
// lumen_depth_to_points_device replaces depthToPointCloud (src/point_cloud.cpp:
// 11-55): every pixel with 0 < Z <= 100 becomes a point
// ((float)((u - cx) Z / fx), (float)((v - cy) Z / fy), Z) in double arithmetic
// like the reference's, coloured from a BGR image (or white), in raster order.
// Three launches: per-row counts, one scan of the counts into row offsets,
// then every row's points written at its offset (warp ballots keep the order
// inside the row).
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

struct __align__(4) ColorLut {
    uint8_t v[768];     // 256 triplets in output channel order
};

__device__ __forceinline__ float disp_depth(int16_t d, float focal, float baseline, float doffs) {
    float z = 0.0f;
    if (d > 0) {
        const float dispFloat = static_cast<float>(d) / 16.0f;
        const float denom = dispFloat + doffs;
        z = (denom > 0.0f) ? ((focal * baseline) / denom) : 0.0f;
    }
    return z;
}

__device__ __forceinline__ int depth_color_index(float z, float minDepth, float maxDepth) {
    if (z <= 0.0f || z > maxDepth * 2) return 0;
    // NaN: the source's fminf(1, NaN) = 1 gives index 0.  Tested on the bits,
    // so that a fast-math lowering of the clamp to a saturate (NaN -> 0,
    // index 255) cannot change it.
    if ((__float_as_uint(z) & 0x7fffffffu) > 0x7f800000u) return 0;
    float n = (z - minDepth) / (maxDepth - minDepth);
    n = fmaxf(0.0f, fminf(1.0f, n));
    n = 1.0f - n;
    return static_cast<int>(n * 255.0f);
}

// Once per CTA, as 32-bit words: the CTAs stride over rows (grid_rows) so
// the staging is paid about eight times per SM, not once per 256 pixels.
__device__ __forceinline__ void stage_lut(const ColorLut& lut, uint8_t* s) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(lut.v);
    uint32_t* dst = reinterpret_cast<uint32_t*>(s);
    for (int i = threadIdx.x; i < 192; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// rows a launch's CTAs stride over: about 8 CTAs of 256 threads per SM
static int grid_rows(int width, int height) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int gx = (width + 255) / 256;
    int gy = (sms * 8 + gx - 1) / gx;
    return gy < height ? gy : height;
}

// COLOR: also writes the colour of each depth (rgb, 3 bytes a pixel); depth
// may then be null.
template <bool COLOR>
__global__ void __launch_bounds__(256)
depth_kernel(const int16_t* __restrict__ disp, size_t dispPitch, int W, int H, float focal,
             float baseline, float doffs, float* __restrict__ depth, size_t depthPitch,
             float minDepth, float maxDepth, const __grid_constant__ ColorLut lut,
             uint8_t* __restrict__ rgb, size_t rgbPitch) {
    __shared__ __align__(4) uint8_t sl[COLOR ? 768 : 4];
    if (COLOR) stage_lut(lut, sl);
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W) return;
    for (int y = blockIdx.y; y < H; y += gridDim.y) {
        const float z = disp_depth(disp[(size_t)y * dispPitch + x], focal, baseline, doffs);
        if (depth) depth[(size_t)y * depthPitch + x] = z;
        if (COLOR) {
            const int c = depth_color_index(z, minDepth, maxDepth) * 3;
            uint8_t* o = rgb + (size_t)y * rgbPitch + (size_t)x * 3;
            o[0] = sl[c];
            o[1] = sl[c + 1];
            o[2] = sl[c + 2];
        }
    }
}

__global__ void __launch_bounds__(256)
colorize_kernel(const float* __restrict__ depth, size_t depthPitch, int W, int H, float minDepth,
                float maxDepth, const __grid_constant__ ColorLut lut, uint8_t* __restrict__ rgb,
                size_t rgbPitch) {
    __shared__ __align__(4) uint8_t sl[768];
    stage_lut(lut, sl);
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W) return;
    for (int y = blockIdx.y; y < H; y += gridDim.y) {
        const int c = depth_color_index(depth[(size_t)y * depthPitch + x], minDepth, maxDepth) * 3;
        uint8_t* o = rgb + (size_t)y * rgbPitch + (size_t)x * 3;
        o[0] = sl[c];
        o[1] = sl[c + 1];
        o[2] = sl[c + 2];
    }
}

// ---- point cloud ----
__device__ __forceinline__ bool point_valid(float z) { return !(z <= 0.0f || z > 100.0f); }

constexpr int kPtThreads = 256;

// rowCount[y] = valid pixels of row y (one CTA a row)
__global__ void __launch_bounds__(kPtThreads)
point_count_kernel(const float* __restrict__ depth, size_t depthPitch, int W, int* __restrict__ rowCount) {
    __shared__ int warpSum[kPtThreads / 32];
    const float* row = depth + (size_t)blockIdx.x * depthPitch;
    int n = 0;
    for (int x = threadIdx.x; x < W; x += kPtThreads) n += point_valid(row[x]);
    n = __reduce_add_sync(0xffffffffu, n);
    if ((threadIdx.x & 31) == 0) warpSum[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kPtThreads / 32; ++w) t += warpSum[w];
        rowCount[blockIdx.x] = t;
    }
}

// in place: off[0..H-1] row counts -> off[0..H] exclusive offsets (one CTA)
__global__ void __launch_bounds__(1024)
point_scan_kernel(int* __restrict__ off, int H) {
    __shared__ int warpSum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < H; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < H ? off[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warpSum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = warpSum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            warpSum[lane] = w;     // inclusive over warps
        }
        __syncthreads();
        const int excl = carry + (warp ? warpSum[warp - 1] : 0) + incl - v;
        if (i < H) off[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[H] = carry;
}

__global__ void __launch_bounds__(kPtThreads)
point_write_kernel(const float* __restrict__ depth, size_t depthPitch, int W,
                   const uint8_t* __restrict__ bgr, size_t bgrPitch, double fx, double fy, double cx,
                   double cy, const int* __restrict__ off, float4* __restrict__ pts) {
    __shared__ int warpSum[kPtThreads / 32];
    const int y = blockIdx.x;
    const float* row = depth + (size_t)y * depthPitch;
    const uint8_t* crow = bgr ? bgr + (size_t)y * bgrPitch : nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int base = off[y];
    const double Yf = ((double)y - cy);
    for (int x0 = 0; x0 < W; x0 += kPtThreads) {
        const int x = x0 + threadIdx.x;
        const float z = x < W ? row[x] : 0.0f;
        const bool ok = x < W && point_valid(z);
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) warpSum[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kPtThreads / 32; ++w) {
            const int c = warpSum[w];
            before += w < warp ? c : 0;
            total += c;
        }
        if (ok) {
            const int at = base + before + __popc(m & ((1u << lane) - 1u));
            float4 p;
            p.x = static_cast<float>(((double)x - cx) * (double)z / fx);
            p.y = static_cast<float>(Yf * (double)z / fy);
            p.z = z;
            unsigned c = 0x00ffffffu;
            if (crow) {
                const uint8_t* q = crow + (size_t)x * 3;
                c = (unsigned)q[2] | ((unsigned)q[1] << 8) | ((unsigned)q[0] << 16);
            }
            p.w = __uint_as_float(c);
            pts[at] = p;
        }
        base += total;
        __syncthreads();
    }
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

static lumen_status launched(const char* who) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(LUMEN_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
    return LUMEN_OK;
}

// 0 = packed; else at least the packed size and a multiple of the element size
static bool fix_stride(size_t& stride, int width, size_t elem) {
    if (!stride) stride = (size_t)width * elem;
    return stride >= (size_t)width * elem && stride % elem == 0;
}

extern "C" lumen_status lumen_disparity_to_depth_color_device(
    const int16_t* d_disp, int width, int height, size_t disp_stride, float focal_px, float baseline,
    float disparity_offset_px, float* d_depth, size_t depth_stride, float min_depth, float max_depth,
    const uint8_t* lut, uint8_t* d_rgb, size_t rgb_stride, void* stream) {
    const char* who = "lumen_disparity_to_depth_color_device";
    if (!d_disp || width <= 0 || height <= 0 || (!d_depth && !d_rgb))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": empty input or no output");
    if (d_rgb && !lut) return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": NULL colour table");
    if (!fix_stride(disp_stride, width, 2) || !fix_stride(depth_stride, width, 4) ||
        !fix_stride(rgb_stride, width, 3))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": bad stride");
    ColorLut t{};
    if (d_rgb) memcpy(t.v, lut, sizeof(t.v));
    const dim3 g((width + 255) / 256, grid_rows(width, height));
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (d_rgb)
        depth_kernel<true><<<g, 256, 0, s>>>(d_disp, disp_stride / 2, width, height, focal_px, baseline,
                                             disparity_offset_px, d_depth, depth_stride / 4, min_depth,
                                             max_depth, t, d_rgb, rgb_stride);
    else
        depth_kernel<false><<<g, 256, 0, s>>>(d_disp, disp_stride / 2, width, height, focal_px, baseline,
                                              disparity_offset_px, d_depth, depth_stride / 4, 0.f, 0.f, t,
                                              nullptr, 0);
    return launched(who);
}

extern "C" lumen_status lumen_disparity_to_depth_device(const int16_t* d_disp, int width, int height,
                                                        size_t disp_stride, float focal_px,
                                                        float baseline, float disparity_offset_px,
                                                        float* d_depth, size_t depth_stride,
                                                        void* stream) {
    if (!d_depth)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, "lumen_disparity_to_depth_device: NULL output");
    return lumen_disparity_to_depth_color_device(d_disp, width, height, disp_stride, focal_px, baseline,
                                                 disparity_offset_px, d_depth, depth_stride, 0.f, 0.f,
                                                 nullptr, nullptr, 0, stream);
}

extern "C" lumen_status lumen_depth_colorize_device(const float* d_depth, int width, int height,
                                                    size_t depth_stride, float min_depth, float max_depth,
                                                    const uint8_t* lut, uint8_t* d_rgb, size_t rgb_stride,
                                                    void* stream) {
    const char* who = "lumen_depth_colorize_device";
    if (!d_depth || !d_rgb || !lut || width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": NULL or empty argument");
    if (!fix_stride(depth_stride, width, 4) || !fix_stride(rgb_stride, width, 3))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": bad stride");
    ColorLut t;
    memcpy(t.v, lut, sizeof(t.v));
    colorize_kernel<<<dim3((width + 255) / 256, grid_rows(width, height)), 256, 0,
                      static_cast<cudaStream_t>(stream)>>>(
        d_depth, depth_stride / 4, width, height, min_depth, max_depth, t, d_rgb, rgb_stride);
    return launched(who);
}

extern "C" lumen_status lumen_depth_to_points_device(const float* d_depth, int width, int height,
                                                     size_t depth_stride, const uint8_t* d_bgr,
                                                     size_t bgr_stride, double fx, double fy, double cx,
                                                     double cy, lumen_point3d* d_points,
                                                     int* d_row_offsets, void* stream) {
    const char* who = "lumen_depth_to_points_device";
    if (!d_depth || !d_points || !d_row_offsets || width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": NULL or empty argument");
    if ((size_t)width * height > (size_t)INT_MAX)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": more than 2^31-1 pixels");
    if (reinterpret_cast<uintptr_t>(d_points) % 16)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": points not 16-byte aligned");
    if (!fix_stride(depth_stride, width, 4) || (d_bgr && !fix_stride(bgr_stride, width, 3)))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": bad stride");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    point_count_kernel<<<height, kPtThreads, 0, s>>>(d_depth, depth_stride / 4, width, d_row_offsets);
    point_scan_kernel<<<1, 1024, 0, s>>>(d_row_offsets, height);
    point_write_kernel<<<height, kPtThreads, 0, s>>>(d_depth, depth_stride / 4, width, d_bgr, bgr_stride,
                                                     fx, fy, cx, cy, d_row_offsets,
                                                     reinterpret_cast<float4*>(d_points));
    return launched(who);
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

extern "C" lumen_status lumen_depth_to_points(const float* depth, int width, int height, size_t depth_stride,
                                              const uint8_t* bgr, size_t bgr_stride, double fx, double fy,
                                              double cx, double cy, lumen_point3d* points, int* count) {
    const char* who = "lumen_depth_to_points";
    if (!depth || !points || !count || width <= 0 || height <= 0)
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": NULL or empty argument");
    if (!fix_stride(depth_stride, width, 4) || (bgr && !fix_stride(bgr_stride, width, 3)))
        return set_error(LUMEN_ERR_INVALID_ARGUMENT, std::string(who) + ": bad stride");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(LUMEN_ERR_NO_DEVICE, "no CUDA device available");
    const size_t n = (size_t)width * height;
    struct Bufs {
        void* p[4] = {nullptr, nullptr, nullptr, nullptr};
        ~Bufs() {
            for (void* q : p)
                if (q) cudaFree(q);
        }
    } b;
    cudaError_t e = cudaMalloc(&b.p[0], depth_stride * height);
    if (e == cudaSuccess && bgr) e = cudaMalloc(&b.p[1], bgr_stride * height);
    if (e == cudaSuccess) e = cudaMalloc(&b.p[2], n * sizeof(lumen_point3d));
    if (e == cudaSuccess) e = cudaMalloc(&b.p[3], (height + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b.p[0], depth, depth_stride * height, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && bgr) e = cudaMemcpy(b.p[1], bgr, bgr_stride * height, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(LUMEN_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
    const lumen_status st = lumen_depth_to_points_device(
        static_cast<const float*>(b.p[0]), width, height, depth_stride, static_cast<const uint8_t*>(b.p[1]),
        bgr_stride, fx, fy, cx, cy, static_cast<lumen_point3d*>(b.p[2]), static_cast<int*>(b.p[3]), nullptr);
    if (st != LUMEN_OK) return st;
    int total = 0;
    e = cudaMemcpy(&total, static_cast<int*>(b.p[3]) + height, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && total > 0)
        e = cudaMemcpy(points, b.p[2], (size_t)total * sizeof(lumen_point3d), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(LUMEN_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
    *count = total;
    return LUMEN_OK;
}
