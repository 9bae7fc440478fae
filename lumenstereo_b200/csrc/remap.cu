// remap.cu -- rectification remap of both images in one launch.
//
// Replaces remapKernelSimple (src/rectification.cu:201-253), launched twice on
// the legacy default stream by StereoRectifier::rectify (:324-340).  Same
// arithmetic (floorf taps, float bilinear weights, out-of-image taps read as
// 0, +0.5 then truncation); compiled with --use_fast_math like the reference,
// so the weighted sum contracts into the same fused multiply-adds.
#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

__global__ void __launch_bounds__(256)
remap_kernel(const uint8_t* __restrict__ srcL, const uint8_t* __restrict__ srcR,
             const float* __restrict__ mxL, const float* __restrict__ myL,
             const float* __restrict__ mxR, const float* __restrict__ myR,
             uint8_t* __restrict__ dstL, uint8_t* __restrict__ dstR, int width, int height,
             int channels) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= width) return;
    const bool right = blockIdx.z != 0;
    const uint8_t* src = right ? srcR : srcL;
    const float* mapX = right ? mxR : mxL;
    const float* mapY = right ? myR : myL;
    uint8_t* dst = right ? dstR : dstL;
    const int idx = y * width + x;
    const float srcXf = mapX[idx];
    const float srcYf = mapY[idx];
    const int x0 = static_cast<int>(floorf(srcXf));
    const int y0 = static_cast<int>(floorf(srcYf));
    const int x1 = x0 + 1;
    const int y1 = y0 + 1;
    const float dx = srcXf - x0;
    const float dy = srcYf - y0;
    const float w00 = (1.0f - dx) * (1.0f - dy);
    const float w01 = (1.0f - dx) * dy;
    const float w10 = dx * (1.0f - dy);
    const float w11 = dx * dy;
    const int rowStride = width * channels;
    const bool valid00 = (x0 >= 0 && x0 < width && y0 >= 0 && y0 < height);
    const bool valid01 = (x0 >= 0 && x0 < width && y1 >= 0 && y1 < height);
    const bool valid10 = (x1 >= 0 && x1 < width && y0 >= 0 && y0 < height);
    const bool valid11 = (x1 >= 0 && x1 < width && y1 >= 0 && y1 < height);
    for (int c = 0; c < channels; c++) {
        const float v00 = valid00 ? static_cast<float>(src[y0 * rowStride + x0 * channels + c]) : 0.0f;
        const float v01 = valid01 ? static_cast<float>(src[y1 * rowStride + x0 * channels + c]) : 0.0f;
        const float v10 = valid10 ? static_cast<float>(src[y0 * rowStride + x1 * channels + c]) : 0.0f;
        const float v11 = valid11 ? static_cast<float>(src[y1 * rowStride + x1 * channels + c]) : 0.0f;
        const float val = w00 * v00 + w01 * v01 + w10 * v10 + w11 * v11;
        dst[y * rowStride + x * channels + c] = static_cast<unsigned char>(val + 0.5f);
    }
}

void launch_remap(const uint8_t* srcL, const uint8_t* srcR, const float* mxL, const float* myL,
                  const float* mxR, const float* myR, uint8_t* dstL, uint8_t* dstR, int W, int H,
                  int channels, int nImages, cudaStream_t s) {
    dim3 g((W + 255) / 256, H, nImages);
    remap_kernel<<<g, 256, 0, s>>>(srcL, srcR, mxL, myL, mxR, myR, dstL, dstR, W, H, channels);
}

}  // namespace lumen
