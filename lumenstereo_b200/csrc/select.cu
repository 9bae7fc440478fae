// select.cu -- disparity selection and post-processing.
//
// select_team_kernel / select_row_kernel replace selectDisparityWTA +
//                selectDisparityRight (src/sgbm_kernels.cu:748-856): the team
//                kernel stages a row tile in shared memory and serves both
//                views from it; the row kernel handles tiles too large for
//                shared memory.
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

constexpr size_t kSelectSmemMax = 227 * 1024;  // opt-in shared memory per block on sm_100

template <int KS>
static cudaError_t launch_select_team(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W,
                                      int H, int D, int Dp, int minD, int UR, int16_t* dispL,
                                      int16_t* dispR, cudaStream_t s, bool* launched) {
    int T = 0;
    size_t smem = 0;
    for (int t : {128, 64, 32}) {
        const size_t b = (size_t)(t + D - 1) * (Dp + 2) * 2;
        if (b <= kSelectSmemMax) { T = t; smem = b; break; }
    }
    *launched = false;
    // a tile stages T + D - 1 pixels for T outputs: past ~2.5x re-reads the row
    // kernel, which reads every vector once, is faster
    if (T == 0 || 2 * (T + D - 1) > 5 * T) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(select_team_kernel<KS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 g((W + minD + T - 1) / T, H);
    select_team_kernel<KS><<<g, 256, smem, s>>>(agg, aggB, wrap, W, D, Dp, minD, UR, T, dispL, dispR);
    *launched = true;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// select_row_kernel: both selections for one image row per CTA (the
// fallback when a tile of the team kernel does not fit in shared memory):
// each aggregated vector is read once; the left view is a warp per pixel
// with lane l holding d = l + 32 j, the right view a shared-memory
// atomicMin over (cost << 16 | d) keys of right pixel xr = x - minD - d
// (ties to the smaller d), whose subpixel neighbours are then read at the left
// pixel xr + minD + bestD (src/sgbm_kernels.cu:839-845).
// ---------------------------------------------------------------------------
template <int NJ>
__global__ void __launch_bounds__(256)
select_row_kernel(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB, int W,
                  int D, int Dp, int minD, int UR, int16_t* __restrict__ dispL,
                  int16_t* __restrict__ dispR) {
    extern __shared__ uint32_t rec[];  // [W] right-view keys
    const int y = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < W; i += blockDim.x) rec[i] = 0xFFFFFFFFu;
    __syncthreads();
    const uint16_t* rowA = agg + (size_t)y * W * Dp;
    const uint16_t* rowB = aggB ? aggB + (size_t)y * W * Dp : nullptr;
    auto cost_at = [&](int x, int d) -> uint32_t {
        const size_t i = (size_t)x * Dp + d;
        uint32_t c = rowA[i];
        if (rowB) c = (c + rowB[i]) & 0xFFFFu;
        return c;
    };
    for (int x = warp; x < W; x += nw) {
        uint32_t key[NJ];
        uint32_t kl = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int d = lane + 32 * j;
            uint32_t k = 0xFFFFFFFFu;
            if (d < D) k = (cost_at(x, d) << 16) | (uint32_t)d;
            key[j] = k;
            kl = min(kl, k);
        }
        const uint32_t kmin = __reduce_min_sync(kFullMask, kl);
        const uint32_t best = kmin >> 16;
        const int bestD = (int)(kmin & 0xFFFFu);
        uint32_t m2 = 0xFFFFu;
#pragma unroll
        for (int j = 0; j < NJ; ++j)
            if (key[j] != 0xFFFFFFFFu && (int)(key[j] & 0xFFFFu) != bestD) m2 = min(m2, key[j] >> 16);
        const uint32_t second = __reduce_min_sync(kFullMask, m2);
        if (lane == 0) {
            int16_t out;
            if (UR > 0 && second != 0xFFFFu && second <= best + (best * (uint32_t)UR) / 100u) {
                out = -1;
            } else if (bestD > 0 && bestD < D - 1) {
                out = subpixel_disp((float)cost_at(x, bestD - 1), (float)best, (float)cost_at(x, bestD + 1),
                                    bestD, D, minD);
            } else {
                out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
            }
            dispL[(size_t)y * W + x] = out;
        }
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int xr = x - minD - (lane + 32 * j);
            if (key[j] != 0xFFFFFFFFu && xr >= 0) atomicMin(&rec[xr], key[j]);
        }
    }
    __syncthreads();
    for (int xr = threadIdx.x; xr < W; xr += blockDim.x) {
        const uint32_t k = rec[xr];
        const int bestD = k == 0xFFFFFFFFu ? 0 : (int)(k & 0xFFFFu);
        int16_t out;
        if (bestD > 0 && bestD < D - 1) {
            const int lx = xr + minD + bestD;
            out = subpixel_disp((float)cost_at(lx, bestD - 1), (float)(k >> 16), (float)cost_at(lx, bestD + 1),
                                bestD, D, minD);
        } else {
            out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
        }
        dispR[(size_t)y * W + xr] = out;
    }
}

template <int NJ>
static cudaError_t launch_select_row(const uint16_t* agg, const uint16_t* aggB, int W, int H, int D,
                                     int Dp, int minD, int UR, int16_t* dispL, int16_t* dispR,
                                     cudaStream_t s) {
    const size_t smem = (size_t)W * 4;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(select_row_kernel<NJ>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    select_row_kernel<NJ><<<H, 256, smem, s>>>(agg, aggB, W, D, Dp, minD, UR, dispL, dispR);
    return cudaGetLastError();
}

bool select_needs_summed_volume(int D, int Dp) {
    (void)D;
    (void)Dp;
    return false;  // both select kernels sum the two partial volumes themselves
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
    // the row kernel sums uint16 values mod 2^16 whether or not they can wrap
    if ((size_t)W * 4 > kSelectSmemMax) return cudaErrorInvalidValue;
    switch (Dp / 32) {
    case 2: return launch_select_row<2>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 4: return launch_select_row<4>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 6: return launch_select_row<6>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 8: return launch_select_row<8>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 10: return launch_select_row<10>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 12: return launch_select_row<12>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 14: return launch_select_row<14>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
    case 16: return launch_select_row<16>(agg, aggB, W, H, D, Dp, minD, UR, dispL, dispR, s);
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
    // positive-only upper median (src/sgbm_kernels.cu:892-935): non-positive
    // neighbours become +32767 (above every valid 1/16-px disparity), a
    // min/max network sorts the nine values in registers, and the
    // count/2-th positive value is picked
    int v[9];
    int count = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int val = M[cy + dy][cx + dx];
            const bool pos = val > 0;
            count += pos;
            v[(dy + 1) * 3 + dx + 1] = pos ? val : 32767;
        }
    auto cx2 = [](int& a, int& b) { const int lo = min(a, b); b = max(a, b); a = lo; };
    // 9-input sorting network (25 compare-exchanges)
    cx2(v[0], v[1]); cx2(v[3], v[4]); cx2(v[6], v[7]);
    cx2(v[1], v[2]); cx2(v[4], v[5]); cx2(v[7], v[8]);
    cx2(v[0], v[1]); cx2(v[3], v[4]); cx2(v[6], v[7]);
    cx2(v[0], v[3]); cx2(v[3], v[6]); cx2(v[0], v[3]);
    cx2(v[1], v[4]); cx2(v[4], v[7]); cx2(v[1], v[4]);
    cx2(v[2], v[5]); cx2(v[5], v[8]); cx2(v[2], v[5]);
    cx2(v[1], v[3]); cx2(v[5], v[7]); cx2(v[2], v[6]);
    cx2(v[4], v[6]); cx2(v[2], v[4]); cx2(v[2], v[3]);
    cx2(v[5], v[6]);
    const int k = count >> 1;
    int med = v[0];
    med = k == 1 ? v[1] : med;
    med = k == 2 ? v[2] : med;
    med = k == 3 ? v[3] : med;
    med = k == 4 ? v[4] : med;
    out[(size_t)y * outPitch + x] = count == 0 ? M[cy][cx] : (int16_t)med;
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
