// select.cu -- disparity selection and post-processing.
//
// select_slide_kernel replaces selectDisparityWTA + selectDisparityRight
//                (src/sgbm_kernels.cu:748-856): both views in one read of
//                the aggregated volume.
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
// select_slide_kernel: both selections in ONE read of every aggregated vector.
// A CTA owns an image row; teams of TL lanes walk contiguous segments of it
// pixel by pixel, a lane holding M = 2*KS consecutive disparities of the
// pixel (the sum of the two partial volumes).
//  * left view: every element becomes a key (cost << 16 | d); the two
//    smallest keys of the pixel (lane pairs merged by an xor butterfly) give
//    the minimum, its first index (ties to the smaller d, like the
//    reference's strict < scan, src/sgbm_kernels.cu:764-777) and the second
//    order statistic (the min with that one element removed);
//  * right view: right pixel xr collects keys from (x, d) with x - d =
//    xr + minD, a diagonal of the volume.  The team keeps a sliding array of
//    M*TL partial minima, slot d standing for xr = x - minD - d: stepping to
//    x + 1 moves every slot up by one (in registers: the loop is unrolled M
//    times, the physical register of a slot rotates with the step, and only
//    the slot that crosses into the next lane moves, by one shuffle), then
//    takes the min with the new pixel's keys.  The slot that leaves the top
//    of the team holds a complete right pixel; it and the partial slots at a
//    segment's two ends go to a row array in shared memory by atomicMin.
// Subpixel neighbours (the costs at d - 1 and d + 1 of the winning pixel's
// own vector) travel with the keys when NB: every element carries the
// packed pair (c[d-1] << 16 | c[d+1]), taken from the lane's registers and
// one shuffle from each neighbouring lane; a slot or a left-view minimum
// that takes a key takes its pair, and the row array holds 64-bit
// (key << 32 | pair) records.  Nothing is re-read, so the volumes cross
// HBM once.  Without NB (lanes of more than 8 words, or rows too wide
// for 8 bytes a pixel of shared memory) the neighbours are re-read from the
// volumes.  The 1/16-px
// outputs equal the reference's bit for bit either way.
// ---------------------------------------------------------------------------
// w = a + b (+ c + d when NV == 4) over a lane's KS words (mod 2^16 per half when wrap)
__device__ __forceinline__ uint32_t vsum(uint32_t x, uint32_t y, bool wrap) { return wrap ? __vadd2(x, y) : x + y; }

template <int KS, int NV>
__device__ __forceinline__ void slide_load(const uint16_t* __restrict__ a, const uint16_t* __restrict__ b,
                                           const uint16_t* __restrict__ c, const uint16_t* __restrict__ d,
                                           bool wrap, uint32_t (&w)[KS]) {
    if constexpr (KS % 4 == 0) {
#pragma unroll
        for (int i = 0; i < KS / 4; ++i) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(a) + i);
            if (NV == 4 || b) {
                const uint4 u = __ldg(reinterpret_cast<const uint4*>(b) + i);
                v = make_uint4(vsum(v.x, u.x, wrap), vsum(v.y, u.y, wrap), vsum(v.z, u.z, wrap), vsum(v.w, u.w, wrap));
            }
            if (NV == 4) {
                const uint4 u = __ldg(reinterpret_cast<const uint4*>(c) + i);
                const uint4 q = __ldg(reinterpret_cast<const uint4*>(d) + i);
                v = make_uint4(vsum(v.x, vsum(u.x, q.x, wrap), wrap), vsum(v.y, vsum(u.y, q.y, wrap), wrap),
                               vsum(v.z, vsum(u.z, q.z, wrap), wrap), vsum(v.w, vsum(u.w, q.w, wrap), wrap));
            }
            w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
        }
    } else {
        static_assert(KS % 2 == 0, "lanes hold an even number of words");
#pragma unroll
        for (int i = 0; i < KS / 2; ++i) {
            uint2 v = __ldg(reinterpret_cast<const uint2*>(a) + i);
            if (NV == 4 || b) {
                const uint2 u = __ldg(reinterpret_cast<const uint2*>(b) + i);
                v = make_uint2(vsum(v.x, u.x, wrap), vsum(v.y, u.y, wrap));
            }
            if (NV == 4) {
                const uint2 u = __ldg(reinterpret_cast<const uint2*>(c) + i);
                const uint2 q = __ldg(reinterpret_cast<const uint2*>(d) + i);
                v = make_uint2(vsum(v.x, vsum(u.x, q.x, wrap), wrap), vsum(v.y, vsum(u.y, q.y, wrap), wrap));
            }
            w[2 * i] = v.x; w[2 * i + 1] = v.y;
        }
    }
}

template <int NV>
__device__ __forceinline__ uint32_t vol_cost(const uint16_t* __restrict__ a, const uint16_t* __restrict__ b,
                                             const uint16_t* __restrict__ c, const uint16_t* __restrict__ d,
                                             size_t i) {
    uint32_t v = __ldg(a + i);
    if (NV == 4 || b) v += __ldg(b + i);
    if (NV == 4) v += (uint32_t)__ldg(c + i) + __ldg(d + i);
    return v & 0xFFFFu;
}

// Shared-memory ring of the staged pixels (PF > 0): per slot, volume and
// 16-byte quarter of a lane's words, one uint4 a thread (consecutive threads
// consecutive uint4, so a warp's loads hit distinct banks).
__host__ __device__ inline size_t select_ring_bytes(int PF, int NV, int KS) {
    return (size_t)PF * NV * (KS / 4) * 256 * 16;
}
constexpr int kSelL2Ahead = 3;   // pixels of L2 prefetch ahead (register form)
__device__ __forceinline__ void sel_prefetch_l2(const void* gmem) {
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(gmem));
}
__device__ __forceinline__ void sel_cp16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

// PF = 0: the next pixel's words are loaded into registers one pixel ahead.
// PF = 2 or 3 (needs KS % 4 == 0): each thread copies its words of pixel
// x + PF - 1 into a PF-slot shared ring with cp.async while it works on pixel
// x, so PF - 1 pixels of every team are in flight and the registers hold only
// summed words.  The launcher takes it where it measured faster (4-word
// lanes); with 8-word lanes the register form's loads stall the warps (4
// cycles per issued instruction) but the staged form was slower still.
template <int TL, int KS, bool FULL, int NV, bool NB, int PF = 0>
__device__ __forceinline__ void
select_slide_body(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB,
                  const uint16_t* __restrict__ aggC, const uint16_t* __restrict__ aggD, int wrap,
                  int W, int D, int Dp, int minD, int UR, int S, int16_t* __restrict__ dispL,
                  int16_t* __restrict__ dispR) {
    constexpr int M = 2 * KS;
    constexpr uint32_t INF = 0xFFFFFFFFu;
    constexpr unsigned long long INF64 = ~0ull;
    static_assert(PF == 0 || (KS % 4 == 0 && (PF == 2 || PF == 3)), "staged ring");
    extern __shared__ __align__(16) uint32_t rec[];  // [W] right-view keys of the row (then the ring)
    unsigned long long* const rec64 = reinterpret_cast<unsigned long long*>(rec);  // [W] (key << 32 | pair), NB
    const int y = blockIdx.x;
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        if constexpr (NB) rec64[i] = INF64;
        else rec[i] = INF;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int tl = lane & (TL - 1);
    const int xs = (threadIdx.x / TL) * S;
    const int d0 = tl * M;
    const int nv = FULL ? M : min(max(D - d0, 0), M);
    const size_t rowOff = (size_t)y * W * Dp;
    const uint16_t* rowA = agg + rowOff + d0;
    const uint16_t* rowB = aggB ? aggB + rowOff + d0 : nullptr;
    const uint16_t* rowC = NV == 4 ? aggC + rowOff + d0 : nullptr;
    const uint16_t* rowD = NV == 4 ? aggD + rowOff + d0 : nullptr;
    uint32_t R[M], N[M];   // slot keys; NB: their neighbour pairs
#pragma unroll
    for (int j = 0; j < M; ++j) R[j] = INF, N[j] = 0;
    uint32_t wn[KS];
    // the staged ring (PF > 0), after the row records
    constexpr int KQ = KS / 4 > 0 ? KS / 4 : 1;
    uint4* const ring = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(rec) +
                                                 (((size_t)W * (NB ? 8 : 4) + 15) & ~(size_t)15));
    const int nvol = NV == 4 ? 4 : (rowB ? 2 : 1);
    auto stage = [&](int j, int slot) {   // pixel xs + j of the segment into ring slot `slot`
        if constexpr (PF > 0) {
            const int x = xs + j;
            if (j < S && x < W) {
                const uint16_t* const src[4] = {rowA, rowB, rowC, rowD};
#pragma unroll
                for (int v = 0; v < (NV == 4 ? 4 : 2); ++v)
                    if (v < nvol)
#pragma unroll
                        for (int q = 0; q < KQ; ++q)
                            sel_cp16(&ring[((slot * NV + v) * KQ + q) * 256 + threadIdx.x],
                                     src[v] + (size_t)x * Dp + 8 * q);
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
    };
    if constexpr (PF > 0) {
#pragma unroll
        for (int k = 0; k < PF - 1; ++k) stage(k, k);
    } else if (xs < W) {
        slide_load<KS, NV>(rowA + (size_t)xs * Dp, rowB ? rowB + (size_t)xs * Dp : nullptr,
                           NV == 4 ? rowC + (size_t)xs * Dp : nullptr, NV == 4 ? rowD + (size_t)xs * Dp : nullptr,
                           wrap, wn);
    }
    int slotNow = 0;   // ring slot of the current pixel (PF > 0)
    for (int s = 0; s < S; s += M) {
#pragma unroll
        for (int u = 0; u < M; ++u) {
            const int x = xs + s + u;
            const bool px = x < W;
            uint32_t w[KS];
            if constexpr (PF > 0) {
                // pixel x + PF - 1 into the slot pixel x - 1 left; then pixel x has landed
                const int slotNext = slotNow == 0 ? PF - 1 : slotNow - 1;
                stage(s + u + PF - 1, slotNext);
                asm volatile("cp.async.wait_group %0;\n" ::"n"(PF - 1) : "memory");
#pragma unroll
                for (int q = 0; q < KQ; ++q) {
                    uint4 v = ring[((slotNow * NV + 0) * KQ + q) * 256 + threadIdx.x];
                    if (nvol > 1) {
                        const uint4 b = ring[((slotNow * NV + 1) * KQ + q) * 256 + threadIdx.x];
                        v = make_uint4(vsum(v.x, b.x, wrap), vsum(v.y, b.y, wrap), vsum(v.z, b.z, wrap),
                                       vsum(v.w, b.w, wrap));
                    }
                    if (NV == 4) {
                        const uint4 c = ring[((slotNow * NV + 2) * KQ + q) * 256 + threadIdx.x];
                        const uint4 d = ring[((slotNow * NV + 3) * KQ + q) * 256 + threadIdx.x];
                        v = make_uint4(vsum(v.x, vsum(c.x, d.x, wrap), wrap), vsum(v.y, vsum(c.y, d.y, wrap), wrap),
                                       vsum(v.z, vsum(c.z, d.z, wrap), wrap), vsum(v.w, vsum(c.w, d.w, wrap), wrap));
                    }
                    w[4 * q] = v.x; w[4 * q + 1] = v.y; w[4 * q + 2] = v.z; w[4 * q + 3] = v.w;
                }
                slotNow = slotNow + 1 == PF ? 0 : slotNow + 1;
            } else {
#pragma unroll
                for (int k = 0; k < KS; ++k) w[k] = wn[k];
                // the team's pixel three ahead into L2 (one 128-byte line a request,
                // every fourth lane of a team for lanes of 8 words): the register
                // load-ahead of the next pixel then comes from L2
                if (x + kSelL2Ahead < W && (s + u + kSelL2Ahead) < S && (tl * M * 2) % 128 == 0) {
                    const size_t o = (size_t)(x + kSelL2Ahead) * Dp;
                    sel_prefetch_l2(rowA + o);
                    if (rowB) sel_prefetch_l2(rowB + o);
                    if (NV == 4) {
                        sel_prefetch_l2(rowC + o);
                        sel_prefetch_l2(rowD + o);
                    }
                }
                if (x + 1 < W && (s + u + 1) < S)
                    slide_load<KS, NV>(rowA + (size_t)(x + 1) * Dp, rowB ? rowB + (size_t)(x + 1) * Dp : nullptr,
                                       NV == 4 ? rowC + (size_t)(x + 1) * Dp : nullptr,
                                       NV == 4 ? rowD + (size_t)(x + 1) * Dp : nullptr, wrap, wn);
            }
            // slide by one: the slot leaving this lane (logical M-1, physical
            // (M-1-u) mod M) enters the next lane as its logical slot 0 and
            // this lane's logical 0 takes the previous lane's
            const int q = (M - 1 - u + M) % M;
            const uint32_t leaving = R[q];
            const uint32_t incoming = __shfl_up_sync(kFullMask, leaving, 1, TL);
            R[q] = tl == 0 ? INF : incoming;
            if constexpr (NB) N[q] = __shfl_up_sync(kFullMask, N[q], 1, TL);
            // NB: the words holding d0 - 1 (previous lane) and d0 + M (next lane)
            uint32_t prevW = 0, nextW = 0;
            if constexpr (NB) {
                prevW = __shfl_up_sync(kFullMask, w[KS - 1], 1, TL);
                nextW = __shfl_down_sync(kFullMask, w[0], 1, TL);
            }
            const uint32_t pxmask = px ? 0u : INF;
            uint32_t k1 = INF, k2 = INF, n1 = 0;
#pragma unroll
            for (int j = 0; j < M; ++j) {
                const uint32_t c = (j & 1) ? (w[j >> 1] & 0xFFFF0000u) : (w[j >> 1] << 16);
                uint32_t key = (c + (uint32_t)(d0 + j)) | pxmask;
                if (!FULL) key |= (j < nv) ? 0u : INF;
                const int p = ((j - u - 1) % M + M) % M;  // logical j after the slide
                if constexpr (NB) {
                    // (c[d-1] << 16 | c[d+1]): odd j sits in the high half of its word
                    const int i = j >> 1;
                    const uint32_t nb = (j & 1) ? __byte_perm(w[i], i + 1 < KS ? w[i + 1] : nextW, 0x1054)
                                                : __byte_perm(i > 0 ? w[i - 1] : prevW, w[i], 0x3276);
                    const bool lt = key < R[p];
                    R[p] = lt ? key : R[p];
                    N[p] = lt ? nb : N[p];
                    const bool l1 = key < k1;
                    k2 = min(k2, max(k1, key));
                    n1 = l1 ? nb : n1;
                    k1 = l1 ? key : k1;
                } else {
                    R[p] = min(R[p], key);
                    k2 = min(k2, max(k1, key));
                    k1 = min(k1, key);
                }
            }
            // complete right pixel: the top slot of the team
            if (tl == TL - 1) {
                const int xr = x - minD - (M * TL - 1);
                const int top = (M - 1 - u - 1 + 2 * M) % M;
                if (xr >= 0 && xr < W) {
                    if constexpr (NB) {
                        if (R[top] != INF) atomicMin(&rec64[xr], ((unsigned long long)R[top] << 32) | N[top]);
                    } else {
                        atomicMin(&rec[xr], R[top]);
                    }
                }
            }
            // left view: merge the lanes' two smallest keys
#pragma unroll
            for (int o = TL / 2; o >= 1; o >>= 1) {
                const uint32_t b1 = __shfl_xor_sync(kFullMask, k1, o);
                const uint32_t b2 = __shfl_xor_sync(kFullMask, k2, o);
                if constexpr (NB) {
                    const uint32_t bn = __shfl_xor_sync(kFullMask, n1, o);
                    n1 = b1 < k1 ? bn : n1;
                }
                k2 = min(max(k1, b1), min(k2, b2));
                k1 = min(k1, b1);
            }
            if (tl == 0 && px) {
                const uint32_t best = k1 >> 16, second = k2 >> 16;
                const int bestD = (int)(k1 & 0xFFFFu);
                int16_t out;
                if (UR > 0 && second != 0xFFFFu && second <= best + (best * (uint32_t)UR) / 100u) {
                    out = -1;
                } else if (NB && bestD > 0 && bestD < D - 1) {
                    out = subpixel_disp((float)(n1 >> 16), (float)best, (float)(n1 & 0xFFFFu), bestD, D, minD);
                } else if (bestD > 0 && bestD < D - 1) {
                    const size_t i0 = rowOff + (size_t)x * Dp + bestD;
                    out = subpixel_disp((float)vol_cost<NV>(agg, aggB, aggC, aggD, i0 - 1), (float)best,
                                        (float)vol_cost<NV>(agg, aggB, aggC, aggD, i0 + 1), bestD, D, minD);
                } else {
                    out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
                }
                dispL[(size_t)y * W + x] = out;
            }
        }
    }
    // the partial slots at the segment's end (S is a multiple of M, so the
    // rotation is back at phase 0: logical j is physical j)
    {
        const int xe = xs + S - 1;
#pragma unroll
        for (int j = 0; j < M; ++j) {
            const int xr = xe - minD - (d0 + j);
            if (R[j] != INF && xr >= 0 && xr < W) {
                if constexpr (NB) atomicMin(&rec64[xr], ((unsigned long long)R[j] << 32) | N[j]);
                else atomicMin(&rec[xr], R[j]);
            }
        }
    }
    __syncthreads();
    for (int xr = threadIdx.x; xr < W; xr += blockDim.x) {
        const uint32_t k = NB ? (uint32_t)(rec64[xr] >> 32) : rec[xr];
        const int bestD = k == INF ? 0 : (int)(k & 0xFFFFu);
        int16_t out;
        if (NB && bestD > 0 && bestD < D - 1) {
            const uint32_t nb = (uint32_t)rec64[xr];
            out = subpixel_disp((float)(nb >> 16), (float)(k >> 16), (float)(nb & 0xFFFFu), bestD, D, minD);
        } else if (bestD > 0 && bestD < D - 1) {
            const size_t i0 = rowOff + (size_t)(xr + minD + bestD) * Dp + bestD;
            out = subpixel_disp((float)vol_cost<NV>(agg, aggB, aggC, aggD, i0 - 1), (float)(k >> 16),
                                (float)vol_cost<NV>(agg, aggB, aggC, aggD, i0 + 1), bestD, D, minD);
        } else {
            out = subpixel_disp(0.f, 0.f, 0.f, bestD, D, minD);
        }
        dispR[(size_t)y * W + xr] = out;
    }
}

// Neighbours re-read: the compiler's own register budget.
template <int TL, int KS, bool FULL, int NV>
__global__ void __launch_bounds__(256)
select_slide_kernel(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB,
                    const uint16_t* __restrict__ aggC, const uint16_t* __restrict__ aggD, int wrap,
                    int W, int D, int Dp, int minD, int UR, int S, int16_t* __restrict__ dispL,
                    int16_t* __restrict__ dispR) {
    select_slide_body<TL, KS, FULL, NV, false>(agg, aggB, aggC, aggD, wrap, W, D, Dp, minD, UR, S, dispL, dispR);
}

// Neighbours carried: two CTAs an SM with 128 registers for the words and their pairs
// (measured faster than the default budget).
template <int TL, int KS, bool FULL, int NV, int PF>
__global__ void __launch_bounds__(256, 2)
select_slide_nb_kernel(const uint16_t* __restrict__ agg, const uint16_t* __restrict__ aggB,
                       const uint16_t* __restrict__ aggC, const uint16_t* __restrict__ aggD, int wrap,
                       int W, int D, int Dp, int minD, int UR, int S, int16_t* __restrict__ dispL,
                       int16_t* __restrict__ dispR) {
    select_slide_body<TL, KS, FULL, NV, true, PF>(agg, aggB, aggC, aggD, wrap, W, D, Dp, minD, UR, S, dispL, dispR);
}

constexpr size_t kSelectSmemMax = 227 * 1024;  // opt-in shared memory per block on sm_100

template <int TL, int KS>
static cudaError_t launch_select_slide(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W, int H,
                                       int D, int Dp, int minD, int UR, int16_t* dispL, int16_t* dispR,
                                       cudaStream_t s, const uint16_t* aggC, const uint16_t* aggD) {
    constexpr int M = 2 * KS, kTeams = 256 / TL;
    const int seg = (W + kTeams - 1) / kTeams;
    const int S = (seg + M - 1) / M * M;
    // 64-bit row records fit; wider lanes keep re-reading (measured: with 10 words a
    // lane the registers of the pairs cost more than the re-reads save)
    const bool nb = KS <= 8 && (size_t)W * 8 <= kSelectSmemMax;
    const bool four = aggB && aggC && aggD;
    size_t smem = (size_t)W * (nb ? 8 : 4);
    // the staged ring for lanes of 4 words (640x480 D64: selection + post 0.088 ->
    // 0.057 ms): three slots (two pixels in flight) when two CTAs an SM still fit,
    // else two; lanes of 8 words keep the register form (1080p D128: 0.525 ms
    // against 0.695 staged)
    int pf = 0;
    if (nb && KS == 4) {
        const size_t base = (smem + 15) & ~(size_t)15;
        for (int cand : {3, 2})
            if (!pf && 2 * (base + select_ring_bytes(cand, four ? 4 : 2, KS) + 1024) <= 228 * 1024) pf = cand;
        if (pf) smem = base + select_ring_bytes(pf, four ? 4 : 2, KS);
    }
    void (*kern)(const uint16_t*, const uint16_t*, const uint16_t*, const uint16_t*, int, int, int, int, int, int,
                 int, int16_t*, int16_t*);
    if constexpr (KS <= 8) {
        constexpr int P3 = KS == 4 ? 3 : 0, P2 = KS == 4 ? 2 : 0;
        auto pick = [&](auto full3_4, auto part3_4, auto full3_2, auto part3_2) {
            return four ? (D == Dp ? full3_4 : part3_4) : (D == Dp ? full3_2 : part3_2);
        };
        if (!nb)
            kern = pick(select_slide_kernel<TL, KS, true, 4>, select_slide_kernel<TL, KS, false, 4>,
                        select_slide_kernel<TL, KS, true, 2>, select_slide_kernel<TL, KS, false, 2>);
        else if (pf == 3)
            kern = pick(select_slide_nb_kernel<TL, KS, true, 4, P3>, select_slide_nb_kernel<TL, KS, false, 4, P3>,
                        select_slide_nb_kernel<TL, KS, true, 2, P3>, select_slide_nb_kernel<TL, KS, false, 2, P3>);
        else if (pf == 2)
            kern = pick(select_slide_nb_kernel<TL, KS, true, 4, P2>, select_slide_nb_kernel<TL, KS, false, 4, P2>,
                        select_slide_nb_kernel<TL, KS, true, 2, P2>, select_slide_nb_kernel<TL, KS, false, 2, P2>);
        else
            kern = pick(select_slide_nb_kernel<TL, KS, true, 4, 0>, select_slide_nb_kernel<TL, KS, false, 4, 0>,
                        select_slide_nb_kernel<TL, KS, true, 2, 0>, select_slide_nb_kernel<TL, KS, false, 2, 0>);
    } else
        kern = four ? (D == Dp ? select_slide_kernel<TL, KS, true, 4> : select_slide_kernel<TL, KS, false, 4>)
                    : (D == Dp ? select_slide_kernel<TL, KS, true, 2> : select_slide_kernel<TL, KS, false, 2>);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<H, 256, smem, s>>>(agg, aggB, four ? aggC : nullptr, four ? aggD : nullptr, wrap ? 1 : 0, W, D, Dp,
                              minD, UR, S, dispL, dispR);
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
                          cudaStream_t s, const uint16_t* aggC, const uint16_t* aggD) {
    if ((size_t)W * 4 > kSelectSmemMax) return cudaErrorInvalidValue;  // W > 58112: no row array
    switch (Dp / 64) {
    case 1: return launch_select_slide<8, 4>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 2: return launch_select_slide<8, 8>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 3: return launch_select_slide<8, 12>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    // wider pixels spread over 16 lanes: 16-20 words per lane cost occupancy
    case 4: return launch_select_slide<16, 8>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 5: return launch_select_slide<16, 10>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 6: return launch_select_slide<16, 12>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 7: return launch_select_slide<16, 14>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
    case 8: return launch_select_slide<16, 16>(agg, aggB, wrap, W, H, D, Dp, minD, UR, dispL, dispR, s, aggC, aggD);
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
