// ref_harness.cu -- host driver for LumenStereo's own CUDA kernels.
//
// TEST INFRASTRUCTURE ONLY (the GPU-side oracle).  oracle/Makefile compiles
// this file together with the reference's unmodified src/sgbm_kernels.cu and
// remapKernelSimple (src/rectification.cu:201-253), taken from the read-only
// reference tree at build time, into oracle/_ref/libref_sgbm.so.  The
// reference's own host code (src/sgbm_gpu.cu) cannot be built here because it
// includes OpenCV headers, so this driver restates it launch for launch: the
// same grids, blocks, dynamic shared memory size, stage order, zeroing,
// costScale, disp12MaxDiff*16, min(speckleWindowSize,25), speckleRange*16,
// the per-call L_diag allocation of the 8-path mode and the median's
// device-to-device copy back.  Line numbers cite src/sgbm_gpu.cu.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <algorithm>

namespace stereo {
__global__ void prefilterXSobel(const unsigned char*, unsigned char*, int, int, int);
__global__ void computeCostSAD_naive(const unsigned char*, const unsigned char*, unsigned char*, int, int, int, int, int);
__global__ void computeCostSAD_shared(const unsigned char*, const unsigned char*, unsigned char*, int, int, int, int, int);
__global__ void buildCensus5x5(const unsigned char*, uint32_t*, int, int);
__global__ void computeCostCensus_naive(const uint32_t*, const uint32_t*, unsigned char*, int, int, int, int);
__global__ void aggregateCostHorizontalLR(const unsigned char*, uint16_t*, const unsigned char*, int, int, int, int, int, int);
__global__ void aggregateCostHorizontalRL(const unsigned char*, uint16_t*, const unsigned char*, int, int, int, int, int, int);
__global__ void aggregateCostVerticalTB(const unsigned char*, uint16_t*, const unsigned char*, int, int, int, int, int, int);
__global__ void aggregateCostVerticalBT(const unsigned char*, uint16_t*, const unsigned char*, int, int, int, int, int, int);
__global__ void aggregateCostDiagonalTLBR(const unsigned char*, uint16_t*, uint16_t*, const unsigned char*, int, int, int, int, int, int, int);
__global__ void aggregateCostDiagonalBRTL(const unsigned char*, uint16_t*, uint16_t*, const unsigned char*, int, int, int, int, int, int, int);
__global__ void aggregateCostDiagonalTRBL(const unsigned char*, uint16_t*, uint16_t*, const unsigned char*, int, int, int, int, int, int, int);
__global__ void aggregateCostDiagonalBLTR(const unsigned char*, uint16_t*, uint16_t*, const unsigned char*, int, int, int, int, int, int, int);
__global__ void selectDisparityWTA(const uint16_t*, int16_t*, int, int, int, int, int);
__global__ void selectDisparityRight(const uint16_t*, int16_t*, int, int, int, int);
__global__ void consistencyCheck(int16_t*, const int16_t*, int, int, int);
__global__ void medianFilter3x3(const int16_t*, int16_t*, int, int);
__global__ void speckleFilter(int16_t*, int, int, int, int);
__global__ void remapKernelSimple(const unsigned char*, const float*, const float*, unsigned char*, int, int, int);
__global__ void disparityToDepthKernel(const int16_t*, float*, int, int, float, float, float);
__global__ void colorizeDepthKernel(const float*, unsigned char*, int, int, float, float);
extern __constant__ unsigned char turboR[256];
extern __constant__ unsigned char turboG[256];
extern __constant__ unsigned char turboB[256];
}  // namespace stereo

// Field order of oracle_params / lumen_stereo_params; external linkage so the
// extern "C" entry points below are exported.
struct RefParams {  // field order of oracle_params / lumen_stereo_params
    int minDisparity, maxDisparity, blockSize, P1, P2, preFilterCap, uniquenessRatio,
        disp12MaxDiff, speckleWindowSize, speckleRange, useGPU, useSharedMemory, numDirections,
        matchingCostMode;
};

struct RefDump {  // host pointers, any may be null
    uint8_t* pref_left;
    uint8_t* pref_right;
    uint32_t* census_left;
    uint32_t* census_right;
    uint8_t* cost;
    uint16_t* agg;
    int16_t* disp_wta;
    int16_t* disp_right;
    int16_t* disp_lr;
};

namespace {

inline int divUp(int a, int b) { return (a + b - 1) / b; }

#define RCHECK(call)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            std::snprintf(g_err, sizeof(g_err), "%s:%d %s", __FILE__, __LINE__,       \
                          cudaGetErrorString(e_));                                    \
            rc = 3;                                                                   \
            goto cleanup;                                                             \
        }                                                                             \
    } while (0)

char g_err[512];

}  // namespace

extern "C" const char* ref_last_error(void) { return g_err; }

// StereoSGBM::compute for one gray pair (src/sgbm_gpu.cu:147-195).  Returns 0
// on success, 1 invalid argument, 2 range limit, 3 CUDA error.  gpu_ms (may be
// null) receives the device time from the first H2D copy to the final
// disparity, the interval getLastComputeTimeMs covers (:177-191), including
// the 8-path L_diag cudaMalloc the reference makes on every call.
extern "C" int ref_sgbm_run(const RefParams* p, const uint8_t* hleft, const uint8_t* hright,
                            int W, int H, int16_t* hdisp, const RefDump* dump,
                            unsigned pathMask, int repeats, float* gpu_ms) {
    using namespace stereo;
    int rc = 0;
    const int D = p->maxDisparity - p->minDisparity;
    if (W <= 0 || H <= 0 || !hleft || !hright) return 1;  // :148-153
    if (D < 1) return 1;                                  // :159-161
    if (D > 512) return 2;                                // :162-166
    if (pathMask == 0) pathMask = p->numDirections >= 8 ? 0xFFu : 0x0Fu;
    const size_t N = (size_t)W * H, ND = N * (size_t)D;
    unsigned char *dL = nullptr, *dR = nullptr, *dLf = nullptr, *dRf = nullptr, *dCost = nullptr;
    uint32_t *dCL = nullptr, *dCR = nullptr;
    uint16_t *dAgg = nullptr, *dDiag = nullptr;
    int16_t *dDisp = nullptr, *dDispR = nullptr, *dTmp = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float best = 0.f;
    // allocateBuffers (:119-145)
    RCHECK(cudaMalloc(&dL, N));
    RCHECK(cudaMalloc(&dR, N));
    RCHECK(cudaMalloc(&dLf, N));
    RCHECK(cudaMalloc(&dRf, N));
    if (p->matchingCostMode == 1) {
        RCHECK(cudaMalloc(&dCL, N * 4));
        RCHECK(cudaMalloc(&dCR, N * 4));
    }
    RCHECK(cudaMalloc(&dCost, ND));
    RCHECK(cudaMalloc(&dAgg, ND * 2));
    RCHECK(cudaMalloc(&dDisp, N * 2));
    RCHECK(cudaMalloc(&dDispR, N * 2));
    RCHECK(cudaMalloc(&dTmp, N * 2));
    RCHECK(cudaStreamCreate(&s));
    RCHECK(cudaEventCreate(&e0));
    RCHECK(cudaEventCreate(&e1));
    if (repeats < 1) repeats = 1;
    for (int it = 0; it < repeats; ++it) {
        RCHECK(cudaEventRecord(e0, s));
        RCHECK(cudaMemset(dAgg, 0, ND * 2));  // allocateBuffers' agg.zero() (:144)
        RCHECK(cudaMemcpy(dL, hleft, N, cudaMemcpyHostToDevice));   // :181
        RCHECK(cudaMemcpy(dR, hright, N, cudaMemcpyHostToDevice));  // :182
        // computeCostVolume (:197-295)
        {
            const int blockRadius = p->blockSize / 2;
            if (p->matchingCostMode == 1) {
                dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
                buildCensus5x5<<<g, b, 0, s>>>(dL, dCL, W, H);
                buildCensus5x5<<<g, b, 0, s>>>(dR, dCR, W, H);
                computeCostCensus_naive<<<g, b, 0, s>>>(dCL, dCR, dCost, W, H, D, p->minDisparity);
            } else {
                dim3 pb(16, 16), pg(divUp(W, 16), divUp(H, 16));
                const int cap = std::max(1, p->preFilterCap);
                prefilterXSobel<<<pg, pb, 0, s>>>(dL, dLf, W, H, cap);
                prefilterXSobel<<<pg, pb, 0, s>>>(dR, dRf, W, H, cap);
                if (p->useSharedMemory) {
                    dim3 b(32, 16), g(divUp(W, 32), divUp(H, 16));
                    const int pad = blockRadius;
                    const int ltw = 32 + 2 * pad, lth = 16 + 2 * pad;
                    const int rtw = 32 + 3 * pad + p->minDisparity + D, rth = 16 + 2 * pad;
                    const size_t smem = (size_t)(ltw * lth + rtw * rth);
                    if (smem <= 48 * 1024) {
                        computeCostSAD_shared<<<g, b, smem, s>>>(dLf, dRf, dCost, W, H, D,
                                                                 p->minDisparity, blockRadius);
                    } else {
                        dim3 nb(16, 16), ng(divUp(W, 16), divUp(H, 16));
                        computeCostSAD_naive<<<ng, nb, 0, s>>>(dLf, dRf, dCost, W, H, D,
                                                               p->minDisparity, blockRadius);
                    }
                } else {
                    dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
                    computeCostSAD_naive<<<g, b, 0, s>>>(dLf, dRf, dCost, W, H, D,
                                                         p->minDisparity, blockRadius);
                }
            }
            RCHECK(cudaGetLastError());
            RCHECK(cudaStreamSynchronize(s));  // :290
        }
        // aggregateCosts (:297-430)
        {
            RCHECK(cudaMemsetAsync(dAgg, 0, ND * 2, s));
            RCHECK(cudaStreamSynchronize(s));
            int costScale;
            if (p->matchingCostMode == 0) costScale = p->blockSize * p->blockSize;
            else costScale = std::max(1, (p->blockSize * p->blockSize * 2 * p->preFilterCap) / 255);
            const int rb = divUp(H, 256), cb = divUp(W, 256);
            if (pathMask & 1u) aggregateCostHorizontalLR<<<rb, 256, 0, s>>>(dCost, dAgg, dL, W, H, D, p->P1, p->P2, costScale);
            if (pathMask & 2u) aggregateCostHorizontalRL<<<rb, 256, 0, s>>>(dCost, dAgg, dL, W, H, D, p->P1, p->P2, costScale);
            if (pathMask & 4u) aggregateCostVerticalTB<<<cb, 256, 0, s>>>(dCost, dAgg, dL, W, H, D, p->P1, p->P2, costScale);
            if (pathMask & 8u) aggregateCostVerticalBT<<<cb, 256, 0, s>>>(dCost, dAgg, dL, W, H, D, p->P1, p->P2, costScale);
            RCHECK(cudaGetLastError());
            if (pathMask & 0xF0u) {
                RCHECK(cudaMalloc(&dDiag, ND * 2));  // per call, as the reference (:360-361)
                const int maxDiag = W + H - 1;
                const int db = divUp(std::max(W, H), 256);
                if (pathMask & 0x10u) {
                    RCHECK(cudaMemsetAsync(dDiag, 0, ND * 2, s));
                    RCHECK(cudaStreamSynchronize(s));
                    for (int dg = 0; dg < maxDiag; ++dg)
                        aggregateCostDiagonalTLBR<<<db, 256, 0, s>>>(dCost, dAgg, dDiag, dL, W, H, D, p->P1, p->P2, costScale, dg);
                }
                if (pathMask & 0x20u) {
                    RCHECK(cudaMemsetAsync(dDiag, 0, ND * 2, s));
                    RCHECK(cudaStreamSynchronize(s));
                    for (int dg = 0; dg < maxDiag; ++dg)
                        aggregateCostDiagonalBRTL<<<db, 256, 0, s>>>(dCost, dAgg, dDiag, dL, W, H, D, p->P1, p->P2, costScale, dg);
                }
                if (pathMask & 0x40u) {
                    RCHECK(cudaMemsetAsync(dDiag, 0, ND * 2, s));
                    RCHECK(cudaStreamSynchronize(s));
                    for (int dg = 0; dg < maxDiag; ++dg)
                        aggregateCostDiagonalTRBL<<<db, 256, 0, s>>>(dCost, dAgg, dDiag, dL, W, H, D, p->P1, p->P2, costScale, dg);
                }
                if (pathMask & 0x80u) {
                    RCHECK(cudaMemsetAsync(dDiag, 0, ND * 2, s));
                    RCHECK(cudaStreamSynchronize(s));
                    for (int dg = 0; dg < maxDiag; ++dg)
                        aggregateCostDiagonalBLTR<<<db, 256, 0, s>>>(dCost, dAgg, dDiag, dL, W, H, D, p->P1, p->P2, costScale, dg);
                }
                RCHECK(cudaGetLastError());
                RCHECK(cudaStreamSynchronize(s));
                RCHECK(cudaFree(dDiag));
                dDiag = nullptr;
            }
            RCHECK(cudaStreamSynchronize(s));  // :425
        }
        // selectDisparity (:432-458)
        {
            dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
            selectDisparityWTA<<<g, b, 0, s>>>(dAgg, dDisp, W, H, D, p->minDisparity, p->uniquenessRatio);
            selectDisparityRight<<<g, b, 0, s>>>(dAgg, dDispR, W, H, D, p->minDisparity);
            RCHECK(cudaGetLastError());
        }
        if (dump && dump->disp_wta && it == 0) {
            RCHECK(cudaStreamSynchronize(s));
            RCHECK(cudaMemcpy(dump->disp_wta, dDisp, N * 2, cudaMemcpyDeviceToHost));
        }
        // postProcess (:460-515)
        {
            dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
            if (p->disp12MaxDiff >= 0)
                consistencyCheck<<<g, b, 0, s>>>(dDisp, dDispR, W, H, p->disp12MaxDiff * 16);
            if (p->speckleWindowSize > 0)
                speckleFilter<<<g, b, 0, s>>>(dDisp, W, H, std::min(p->speckleWindowSize, 25), p->speckleRange * 16);
            RCHECK(cudaGetLastError());
            if (dump && dump->disp_lr && it == 0) {
                RCHECK(cudaStreamSynchronize(s));
                RCHECK(cudaMemcpy(dump->disp_lr, dDisp, N * 2, cudaMemcpyDeviceToHost));
            }
            medianFilter3x3<<<g, b, 0, s>>>(dDisp, dTmp, W, H);
            RCHECK(cudaGetLastError());
            RCHECK(cudaMemcpyAsync(dDisp, dTmp, N * 2, cudaMemcpyDeviceToDevice, s));
        }
        RCHECK(cudaEventRecord(e1, s));
        RCHECK(cudaEventSynchronize(e1));
        {
            float ms = 0.f;
            RCHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (it == 0 || ms < best) best = ms;
        }
    }
    if (gpu_ms) *gpu_ms = best;
    if (hdisp) RCHECK(cudaMemcpy(hdisp, dDisp, N * 2, cudaMemcpyDeviceToHost));
    if (dump) {
        if (dump->pref_left && p->matchingCostMode == 0) RCHECK(cudaMemcpy(dump->pref_left, dLf, N, cudaMemcpyDeviceToHost));
        if (dump->pref_right && p->matchingCostMode == 0) RCHECK(cudaMemcpy(dump->pref_right, dRf, N, cudaMemcpyDeviceToHost));
        if (dump->census_left && dCL) RCHECK(cudaMemcpy(dump->census_left, dCL, N * 4, cudaMemcpyDeviceToHost));
        if (dump->census_right && dCR) RCHECK(cudaMemcpy(dump->census_right, dCR, N * 4, cudaMemcpyDeviceToHost));
        if (dump->cost) RCHECK(cudaMemcpy(dump->cost, dCost, ND, cudaMemcpyDeviceToHost));
        if (dump->agg) RCHECK(cudaMemcpy(dump->agg, dAgg, ND * 2, cudaMemcpyDeviceToHost));
        if (dump->disp_right) RCHECK(cudaMemcpy(dump->disp_right, dDispR, N * 2, cudaMemcpyDeviceToHost));
    }
cleanup:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(dL); cudaFree(dR); cudaFree(dLf); cudaFree(dRf); cudaFree(dCL); cudaFree(dCR);
    cudaFree(dCost); cudaFree(dAgg); cudaFree(dDiag); cudaFree(dDisp); cudaFree(dDispR); cudaFree(dTmp);
    return rc;
}

// rectifyImageGPU's kernel launch (src/rectification.cu:354-411): one image,
// 16x16 blocks, maps W*H floats, interleaved channels.
extern "C" int ref_remap_run(const uint8_t* hsrc, const float* hmx, const float* hmy, uint8_t* hdst,
                             int W, int H, int channels) {
    int rc = 0;
    const size_t n = (size_t)W * H * channels, m = (size_t)W * H;
    unsigned char *ds = nullptr, *dd = nullptr;
    float *dx = nullptr, *dy = nullptr;
    RCHECK(cudaMalloc(&ds, n));
    RCHECK(cudaMalloc(&dd, n));
    RCHECK(cudaMalloc(&dx, m * 4));
    RCHECK(cudaMalloc(&dy, m * 4));
    RCHECK(cudaMemcpy(ds, hsrc, n, cudaMemcpyHostToDevice));
    RCHECK(cudaMemcpy(dx, hmx, m * 4, cudaMemcpyHostToDevice));
    RCHECK(cudaMemcpy(dy, hmy, m * 4, cudaMemcpyHostToDevice));
    RCHECK(cudaMemset(dd, 0, n));
    {
        dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
        stereo::remapKernelSimple<<<g, b>>>(ds, dx, dy, dd, W, H, channels);
    }
    RCHECK(cudaGetLastError());
    RCHECK(cudaDeviceSynchronize());
    RCHECK(cudaMemcpy(hdst, dd, n, cudaMemcpyDeviceToHost));
cleanup:
    cudaFree(ds); cudaFree(dd); cudaFree(dx); cudaFree(dy);
    return rc;
}

// disparityToDepthGPU's launch (src/depth_map.cu:169-187): 16x16 blocks.
extern "C" int ref_depth_run(const int16_t* hdisp, float* hdepth, int W, int H, float focal,
                             float baseline, float doffs) {
    int rc = 0;
    const size_t n = (size_t)W * H;
    int16_t* dd = nullptr;
    float* dz = nullptr;
    RCHECK(cudaMalloc(&dd, n * 2));
    RCHECK(cudaMalloc(&dz, n * 4));
    RCHECK(cudaMemcpy(dd, hdisp, n * 2, cudaMemcpyHostToDevice));
    {
        dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
        stereo::disparityToDepthKernel<<<g, b>>>(dd, dz, W, H, focal, baseline, doffs);
    }
    RCHECK(cudaGetLastError());
    RCHECK(cudaDeviceSynchronize());
    RCHECK(cudaMemcpy(hdepth, dz, n * 4, cudaMemcpyDeviceToHost));
cleanup:
    cudaFree(dd); cudaFree(dz);
    return rc;
}

// colorizeDepthGPU's launch (src/depth_map.cu:205-222): 16x16 blocks, RGB out.
extern "C" int ref_colorize_run(const float* hdepth, uint8_t* hrgb, int W, int H, float minDepth,
                                float maxDepth) {
    int rc = 0;
    const size_t n = (size_t)W * H;
    float* dz = nullptr;
    unsigned char* dc = nullptr;
    RCHECK(cudaMalloc(&dz, n * 4));
    RCHECK(cudaMalloc(&dc, n * 3));
    RCHECK(cudaMemcpy(dz, hdepth, n * 4, cudaMemcpyHostToDevice));
    {
        dim3 b(16, 16), g(divUp(W, 16), divUp(H, 16));
        stereo::colorizeDepthKernel<<<g, b>>>(dz, dc, W, H, minDepth, maxDepth);
    }
    RCHECK(cudaGetLastError());
    RCHECK(cudaDeviceSynchronize());
    RCHECK(cudaMemcpy(hrgb, dc, n * 3, cudaMemcpyDeviceToHost));
cleanup:
    cudaFree(dz); cudaFree(dc);
    return rc;
}

// The reference's colour table as 256 (R, G, B) triplets, read back from the
// device, for callers that pass it to the engine's caller-given table.
extern "C" int ref_turbo_table(uint8_t* out768) {
    int rc = 0;
    uint8_t r[256], g[256], b[256];
    RCHECK(cudaMemcpyFromSymbol(r, stereo::turboR, 256));
    RCHECK(cudaMemcpyFromSymbol(g, stereo::turboG, 256));
    RCHECK(cudaMemcpyFromSymbol(b, stereo::turboB, 256));
    for (int i = 0; i < 256; ++i) {
        out768[3 * i] = r[i];
        out768[3 * i + 1] = g[i];
        out768[3 * i + 2] = b[i];
    }
cleanup:
    return rc;
}
