// select.cu -- disparity selection and post-processing.
//
// select_kernel  replaces selectDisparityWTA + selectDisparityRight
//                (src/sgbm_kernels.cu:748-856): one CTA per (row, tile of T
//                left pixels) stages the aggregated rows it needs in shared
//                memory once and serves both views from there (the right view
//                reads the diagonal agg[y][xr+minD+d][d]).
// post_kernel    replaces consistencyCheck + speckleFilter + medianFilter3x3
//                and the device-to-device copy back (src/sgbm_kernels.cu:
//                862-1013, src/sgbm_gpu.cu:460-515) with one tiled pass.
//
// This file is compiled with --use_fast_math like the reference (its
// CMakeLists.txt:32), so the parabola's (c0 - c2) / denom is the same
// approximate division and the 1/16-px outputs match bit for bit.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

// src/sgbm_kernels.cu:789-804 / :836-855, same expression order.
__device__ __forceinline__ int16_t subpixel_disp(float c0, float c1, float c2, int bestD, int D,
                                                 int minD) {
    float subpixelD = static_cast<float>(bestD);
    if (bestD > 0 && bestD < D - 1) {
        float denom = 2.0f * (c0 + c2 - 2.0f * c1);
        if (fabsf(denom) > 1e-6f) {
            float delta = (c0 - c2) / denom;
            delta = fmaxf(-1.0f, fminf(1.0f, delta));
            subpixelD += delta;
        }
    }
    return static_cast<int16_t>((subpixelD + minD) * 16.0f);
}

// KW: words per lane as in aggregation (lane holds d in [2KW*lane, 2KW*lane+2KW)).
// SMEM: serve the right view from the staged tile (else gather from global).
template <int KW, bool SMEM>
__global__ void __launch_bounds__(256)
select_kernel(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB, int wrap, int W,
              int H, int D, int Dp, int minD, int UR, int T, int16_t* __restrict__ dispL,
              int16_t* __restrict__ dispR) {
    extern __shared__ __align__(16) uint16_t sa[];
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint16_t* row = agg + (size_t)y * W * Dp;
    const int loadHi = min(W, x0 + T + D - 1);
    const int nload = SMEM ? max(0, loadHi - x0) : 0;
    if (SMEM) {
        const uint4* src = reinterpret_cast<const uint4*>(row + (size_t)x0 * Dp);
        uint4* dst = reinterpret_cast<uint4*>(sa);
        const int n16 = nload * Dp / 8;
        if (aggB) {  // two partial volumes (sweep schedule): sum while staging
            const uint4* srcB = reinterpret_cast<const uint4*>(aggB + (size_t)y * W * Dp + (size_t)x0 * Dp);
            for (int i = threadIdx.x; i < n16; i += blockDim.x) {
                const uint4 p = src[i], q = srcB[i];
                dst[i] = wrap ? make_uint4(__vadd2(p.x, q.x), __vadd2(p.y, q.y), __vadd2(p.z, q.z), __vadd2(p.w, q.w))
                              : make_uint4(p.x + q.x, p.y + q.y, p.z + q.z, p.w + q.w);
            }
        } else {
            for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
    }
    const int dBase = 2 * KW * lane;
    // ---- left view: x in [x0, x0+T) ----
    for (int px = warp; px < T; px += nw) {
        const int x = x0 + px;
        if (x >= W) break;
        const uint16_t* v = SMEM ? sa + (size_t)px * Dp : row + (size_t)x * Dp;
        uint32_t m1 = 0x10000u, m2 = 0x10000u, i1 = 0xFFFFu;
#pragma unroll
        for (int j = 0; j < 2 * KW; ++j) {
            const int d = dBase + j;
            if (d < D) {
                const uint32_t c = v[d];
                if (c < m1) { m2 = m1; m1 = c; i1 = d; }
                else if (c < m2) m2 = c;
            }
        }
        const uint32_t key = (m1 <= 0xFFFFu) ? ((m1 << 16) | i1) : 0xFFFFFFFFu;
        const uint32_t kmin = __reduce_min_sync(kFullMask, key);
        const uint32_t best = kmin >> 16;
        const int bestD = (int)(kmin & 0xFFFFu);
        // second order statistic of the multiset = min(all lane seconds,
        // second smallest of the lane minima)
        const uint32_t sA = __reduce_min_sync(kFullMask, m2);
        const unsigned ties = __ballot_sync(kFullMask, m1 == best);
        uint32_t sB;
        if (__popc(ties) >= 2) sB = best;
        else sB = __reduce_min_sync(kFullMask, key == kmin ? 0x10000u : m1);
        uint32_t second = min(min(sA, sB), 0xFFFFu);
        if (lane == 0) {
            int16_t out;
            if (UR > 0 && second != 0xFFFFu &&
                second <= best + (best * (uint32_t)UR) / 100u) {
                out = -1;
            } else if (bestD > 0 && bestD < D - 1) {
                out = subpixel_disp((float)v[bestD - 1], (float)v[bestD], (float)v[bestD + 1],
                                    bestD, D, minD);
            } else {
                out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
            }
            dispL[(size_t)y * W + x] = out;
        }
    }
    // ---- right view: xr in [x0-minD, x0-minD+T) ----
    for (int px = warp; px < T; px += nw) {
        const int xr = x0 - minD + px;
        if (xr < 0) continue;
        if (xr >= W) break;
        uint32_t key = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < 2 * KW; ++j) {
            const int d = dBase + j;
            const int lx = xr + minD + d;  // = x0 + px + d
            if (d < D && lx < W) {
                const uint32_t c = SMEM ? sa[(size_t)(px + d) * Dp + d] : row[(size_t)lx * Dp + d];
                const uint32_t k = (c << 16) | (uint32_t)d;
                key = min(key, k);
            }
        }
        const uint32_t kmin = __reduce_min_sync(kFullMask, key);
        if (lane == 0) {
            const int bestD = kmin == 0xFFFFFFFFu ? 0 : (int)(kmin & 0xFFFFu);
            int16_t out;
            if (bestD > 0 && bestD < D - 1) {
                const uint16_t* v = SMEM ? sa + (size_t)(px + bestD) * Dp
                                         : row + (size_t)(xr + minD + bestD) * Dp;
                out = subpixel_disp((float)v[bestD - 1], (float)v[bestD], (float)v[bestD + 1],
                                    bestD, D, minD);
            } else {
                out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
            }
            dispR[(size_t)y * W + xr] = out;
        }
    }
}

// ---------------------------------------------------------------------------
// select_team_kernel: the same two selections with teams of 8 lanes per pixel
// (4 pixels per warp); a lane owns KS packed uint16x2 words (2*KS
// disparities).  The left view takes the min with __vminu2, the first index
// of the min with __vcmpeq2, and the second order statistic as the min with
// that one element removed (the multiset statistic the reference's running
// second-minimum computes, src/sgbm_kernels.cu:764-777); team reductions are
// 3-step xor butterflies.  The right view gathers agg[y][xr+minD+d][d] from
// the staged tile, rows padded to Dp+2 elements so that the diagonal spreads
// over the shared-memory banks.
// ---------------------------------------------------------------------------
template <int KS>
__global__ void __launch_bounds__(256)
select_team_kernel(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB, int wrap,
                   int W, int D, int Dp, int minD, int UR, int T, int16_t* __restrict__ dispL,
                   int16_t* __restrict__ dispR) {
    extern __shared__ __align__(16) uint16_t sa[];
    const int pitch = Dp + 2;
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * T;
    const int loadHi = min(W, x0 + T + D - 1);
    const int nload = max(0, loadHi - x0);
    {
        const uint4* srcA = reinterpret_cast<const uint4*>(agg + ((size_t)y * W + x0) * Dp);
        const uint4* srcB = aggB ? reinterpret_cast<const uint4*>(aggB + ((size_t)y * W + x0) * Dp) : nullptr;
        const int per = Dp / 8;  // uint4 per pixel
        for (int i = threadIdx.x; i < nload * per; i += blockDim.x) {
            const int px = i / per, q = i - px * per;
            uint4 v = srcA[i];
            if (srcB) {
                const uint4 w = srcB[i];
                v = wrap ? make_uint4(__vadd2(v.x, w.x), __vadd2(v.y, w.y), __vadd2(v.z, w.z), __vadd2(v.w, w.w))
                         : make_uint4(v.x + w.x, v.y + w.y, v.z + w.z, v.w + w.w);
            }
            uint32_t* d = reinterpret_cast<uint32_t*>(sa + (size_t)px * pitch + q * 8);
            d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, tl = lane & 7;
    const int tteam = (threadIdx.x >> 5) * 4 + (lane >> 3);
    const int nTeams = blockDim.x >> 3;
    const int d0 = tl * 2 * KS;
    const int Tr = (T + nTeams - 1) / nTeams * nTeams;  // uniform trip count for all teams
    // ---------------- left view ----------------
    for (int px = tteam; px < Tr; px += nTeams) {
        const int x = x0 + px;
        const bool ok = px < T && x < W;
        const int pxc = ok ? px : 0;
        const uint32_t* v32 = reinterpret_cast<const uint32_t*>(sa + (size_t)pxc * pitch) + tl * KS;
        uint32_t w[KS];
#pragma unroll
        for (int k = 0; k < KS; ++k) {
            uint32_t val = ok && nload > 0 ? v32[k] : 0xFFFFFFFFu;
            if (d0 + 2 * k >= D) val |= 0x0000FFFFu;
            if (d0 + 2 * k + 1 >= D) val |= 0xFFFF0000u;
            w[k] = val;
        }
        uint32_t m = w[0];
#pragma unroll
        for (int k = 1; k < KS; ++k) m = __vminu2(m, w[k]);
        m = min(m & 0xFFFFu, m >> 16);
        m = min(m, __shfl_xor_sync(kFullMask, m, 4));
        m = min(m, __shfl_xor_sync(kFullMask, m, 2));
        m = min(m, __shfl_xor_sync(kFullMask, m, 1));
        const uint32_t best = m, bx2 = best * 0x10001u;
        uint32_t first = 0xFFFFu;
#pragma unroll
        for (int k = KS - 1; k >= 0; --k) {
            const uint32_t eq = __vcmpeq2(w[k], bx2);
            const uint32_t idx = (eq & 0xFFFFu) ? (uint32_t)(d0 + 2 * k)
                                                : ((eq >> 16) ? (uint32_t)(d0 + 2 * k + 1) : 0xFFFFu);
            first = min(first, idx);
        }
        first = min(first, __shfl_xor_sync(kFullMask, first, 4));
        first = min(first, __shfl_xor_sync(kFullMask, first, 2));
        first = min(first, __shfl_xor_sync(kFullMask, first, 1));
        const int bestD = (int)first;
        // second order statistic: min with the element at bestD removed
        uint32_t m2 = 0xFFFFFFFFu;
#pragma unroll
        for (int k = 0; k < KS; ++k) {
            uint32_t val = w[k];
            if (d0 + 2 * k == bestD) val |= 0x0000FFFFu;
            if (d0 + 2 * k + 1 == bestD) val |= 0xFFFF0000u;
            m2 = __vminu2(m2, val);
        }
        m2 = min(m2 & 0xFFFFu, m2 >> 16);
        m2 = min(m2, __shfl_xor_sync(kFullMask, m2, 4));
        m2 = min(m2, __shfl_xor_sync(kFullMask, m2, 2));
        m2 = min(m2, __shfl_xor_sync(kFullMask, m2, 1));
        if (ok && tl == 0) {
            const uint16_t* v = sa + (size_t)px * pitch;
            int16_t out;
            if (UR > 0 && m2 != 0xFFFFu && m2 <= best + (best * (uint32_t)UR) / 100u) {
                out = -1;
            } else if (bestD > 0 && bestD < D - 1) {
                out = subpixel_disp((float)v[bestD - 1], (float)v[bestD], (float)v[bestD + 1],
                                    bestD, D, minD);
            } else {
                out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
            }
            dispL[(size_t)y * W + x] = out;
        }
    }
    // ---------------- right view ----------------
    for (int px = tteam; px < Tr; px += nTeams) {
        const int xr = x0 - minD + px;
        const bool ok = px < T && xr >= 0 && xr < W;
        uint32_t key = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < 2 * KS; ++j) {
            const int d = d0 + j;
            const int lx = x0 + px + d;
            if (ok && d < D && lx < W) {
                const uint32_t c = sa[(size_t)(px + d) * pitch + d];
                key = min(key, (c << 16) | (uint32_t)d);
            }
        }
        key = min(key, __shfl_xor_sync(kFullMask, key, 4));
        key = min(key, __shfl_xor_sync(kFullMask, key, 2));
        key = min(key, __shfl_xor_sync(kFullMask, key, 1));
        if (ok && tl == 0) {
            const int bestD = key == 0xFFFFFFFFu ? 0 : (int)(key & 0xFFFFu);
            int16_t out;
            if (bestD > 0 && bestD < D - 1) {
                const uint16_t* v = sa + (size_t)(px + bestD) * pitch;
                out = subpixel_disp((float)v[bestD - 1], (float)v[bestD], (float)v[bestD + 1],
                                    bestD, D, minD);
            } else {
                out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
            }
            dispR[(size_t)y * W + xr] = out;
        }
    }
}

template <int KS>
static cudaError_t launch_select_team(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W,
                                      int H, int D, int Dp, int minD, int UR, int16_t* dispL,
                                      int16_t* dispR, cudaStream_t s, bool* launched) {
    int T = 0;
    size_t smem = 0;
    for (int t : {128, 64, 32}) {
        const size_t b = (size_t)(t + D - 1) * (Dp + 2) * 2;
        if (b <= 200 * 1024) { T = t; smem = b; break; }
    }
    *launched = false;
    if (T == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(select_team_kernel<KS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 g((W + minD + T - 1) / T, H);
    select_team_kernel<KS><<<g, 256, smem, s>>>(agg, aggB, wrap, W, D, Dp, minD, UR, T, dispL, dispR);
    *launched = true;
    return cudaGetLastError();
}

template <int KW>
static cudaError_t launch_select_kw(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W,
                                    int H, int D, int Dp, int minD, int UR, int16_t* dispL,
                                    int16_t* dispR, cudaStream_t s) {
    // Largest tile whose staged rows fit in shared memory.
    int T = 0;
    size_t smem = 0;
    for (int t : {128, 64, 32, 16}) {
        const size_t b = (size_t)(t + D - 1) * Dp * 2;
        if (b <= 200 * 1024) { T = t; smem = b; break; }
    }
    if (T > 0) {
        cudaError_t e = cudaFuncSetAttribute(select_kernel<KW, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        dim3 g((W + minD + T - 1) / T, H);
        select_kernel<KW, true><<<g, 256, smem, s>>>(agg, aggB, wrap, W, H, D, Dp, minD, UR, T,
                                                     dispL, dispR);
    } else {
        if (aggB) return cudaErrorInvalidValue;  // the caller sums the partials first
        T = 32;
        dim3 g((W + minD + T - 1) / T, H);
        select_kernel<KW, false><<<g, 256, 0, s>>>(agg, nullptr, 0, W, H, D, Dp, minD, UR, T,
                                                   dispL, dispR);
    }
    return cudaGetLastError();
}

bool select_needs_summed_volume(int D, int Dp) {
    if (Dp <= 320)
        for (int t : {128, 64, 32})
            if ((size_t)(t + D - 1) * (Dp + 2) * 2 <= 200 * 1024) return false;
    for (int t : {128, 64, 32, 16})
        if ((size_t)(t + D - 1) * Dp * 2 <= 200 * 1024) return false;
    return true;
}

__global__ void sum_volumes_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                   uint32_t* __restrict__ dst, size_t n2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = __vadd2(a[i], b[i]);
}

void launch_sum_volumes(const uint16_t* a, const uint16_t* b, uint16_t* dst, size_t n,
                        cudaStream_t s) {
    const size_t n2 = n / 2;
    const int blocks = (int)std::min<size_t>((n2 + 255) / 256, 148 * 16);
    sum_volumes_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const uint32_t*>(a),
                                              reinterpret_cast<const uint32_t*>(b),
                                              reinterpret_cast<uint32_t*>(dst), n2);
}

cudaError_t launch_select(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W, int H,
                          int D, int Dp, int minD, int UR, int16_t* dispL, int16_t* dispR,
                          cudaStream_t s) {
    bool launched = false;
    cudaError_t e = cudaSuccess;
    switch (Dp / 16) {
    case 4: e = launch_select_team<4>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, &launched); break;
    case 8: e = launch_select_team<8>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, &launched); break;
    case 12: e = launch_select_team<12>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, &launched); break;
    case 16: e = launch_select_team<16>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, &launched); break;
    case 20: e = launch_select_team<20>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, &launched); break;
    default: break;
    }
    if (e != cudaSuccess || launched) return e;
    switch (Dp / 64) {
    case 1: return launch_select_kw<1>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 2: return launch_select_kw<2>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 3: return launch_select_kw<3>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 4: return launch_select_kw<4>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 5: return launch_select_kw<5>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 6: return launch_select_kw<6>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 7: return launch_select_kw<7>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 8: return launch_select_kw<8>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s);
    default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// LR check (src/sgbm_kernels.cu:862-890) -> speckle filter with snapshot reads
// (:979-1013; the reference reads neighbours in place while other threads
// write, a race; here every neighbour is read from the post-LR map) ->
// positive-only 3x3 upper median (:892-935).  One CTA per 32x8 output tile;
// the LR-checked map is formed for the tile plus a 3-pixel apron in shared
// memory, out-of-image cells hold -32768 so they are never "positive".
// ---------------------------------------------------------------------------
constexpr int kPostW = 32, kPostH = 8, kApron = 3;
constexpr int kAW = kPostW + 2 * kApron, kAH = kPostH + 2 * kApron;

__global__ void __launch_bounds__(256)
post_kernel(const int16_t* __restrict__ dispL, const int16_t* __restrict__ dispR, int W, int H,
            int lrMaxDiff, int speckleSize, int speckleDiff, int16_t* __restrict__ out,
            size_t outPitch, int16_t* __restrict__ dbgLR) {
    __shared__ int16_t A[kAH][kAW];
    __shared__ int16_t B[kAH][kAW];
    const int bx = blockIdx.x * kPostW, by = blockIdx.y * kPostH;
    const int tid = threadIdx.y * kPostW + threadIdx.x;
    for (int i = tid; i < kAH * kAW; i += kPostW * kPostH) {
        const int ly = i / kAW, lx = i % kAW;
        const int gx = bx + lx - kApron, gy = by + ly - kApron;
        int16_t v = -32768;
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            v = dispL[(size_t)gy * W + gx];
            if (lrMaxDiff >= 0 && v > 0) {
                const int xR = gx - v / 16;
                if (xR < 0 || xR >= W) {
                    v = -1;
                } else {
                    const int16_t dR = dispR[(size_t)gy * W + xR];
                    if (dR <= 0 || abs((int)v - (int)dR) > lrMaxDiff) v = -1;
                }
            }
        }
        A[ly][lx] = v;
    }
    __syncthreads();
    int16_t(*M)[kAW] = A;
    if (speckleSize > 0) {
        for (int i = tid; i < kAH * kAW; i += kPostW * kPostH) {
            const int ly = i / kAW, lx = i % kAW;
            int16_t c = A[ly][lx];
            if (ly >= 2 && ly < kAH - 2 && lx >= 2 && lx < kAW - 2 && c > 0) {
                int similar = 0;
#pragma unroll
                for (int dy = -2; dy <= 2; ++dy)
#pragma unroll
                    for (int dx = -2; dx <= 2; ++dx) {
                        const int16_t nv = A[ly + dy][lx + dx];
                        if (nv > 0 && abs((int)c - (int)nv) <= speckleDiff) ++similar;
                    }
                if (similar < speckleSize) c = -1;
            }
            B[ly][lx] = c;
        }
        __syncthreads();
        M = B;
    }
    const int x = bx + threadIdx.x, y = by + threadIdx.y;
    if (x >= W || y >= H) return;
    const int cy = threadIdx.y + kApron, cx = threadIdx.x + kApron;
    if (dbgLR) dbgLR[(size_t)y * W + x] = M[cy][cx];
    int16_t v[9];
    int count = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int16_t val = M[cy + dy][cx + dx];
            if (val > 0) {
                int j = count++;
                while (j > 0 && v[j - 1] > val) { v[j] = v[j - 1]; --j; }
                v[j] = val;
            }
        }
    out[(size_t)y * outPitch + x] = count == 0 ? M[cy][cx] : v[count / 2];
}

cudaError_t launch_post(const int16_t* dispL, const int16_t* dispR, int W, int H, int lrMaxDiff,
                        int speckleSize, int speckleDiff, int16_t* out, size_t outPitchElems,
                        int16_t* dbgLR, cudaStream_t s) {
    dim3 g((W + kPostW - 1) / kPostW, (H + kPostH - 1) / kPostH);
    post_kernel<<<g, dim3(kPostW, kPostH), 0, s>>>(dispL, dispR, W, H, lrMaxDiff, speckleSize,
                                                    speckleDiff, out, outPitchElems, dbgLR);
    return cudaGetLastError();
}

}  // namespace lumen
