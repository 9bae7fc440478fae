// sweep2_kernel.cuh -- SGM aggregation as two fused wavefront sweeps with
// decoupled row warps (schedule 3).
//
// Same regrouping of the reference's eight path kernels
// (src/sgbm_kernels.cu:315-742) as schedule 2:
//   forward sweep  F: LR (x-1,y)  TB (x,y-1)  TLBR (x-1,y-1)  TRBL (x+1,y-1)
//   backward sweep B: RL (x+1,y)  BT (x,y+1)  BRTL (x+1,y+1)  BLTR (x-1,y+1)
// in "sweep coordinates" (u, v): x = u or W-1-u, y = v or H-1-v.  The four
// path vectors of a pixel are summed in registers and stored once per sweep.
//
// Work decomposition:
//  * a band is R consecutive sweep rows; each row is one warp (32 lanes over
//    the disparities, KW packed uint16x2 words per lane) that walks its row
//    pixel by pixel, carrying the horizontal path in registers;
//  * row r hands its TB/TLBR/TRBL vectors (and their minima) to row r+1
//    through a shared-memory ring; the rows run decoupled, synchronised only
//    by per-row progress counters (acquire/release at CTA scope), so a row
//    waits only when its predecessor has not yet produced pixel u+1 or its
//    successor still needs a slot it wants to overwrite;
//  * an import warp copies the previous band's last row from a global
//    exchange row into the band's import ring as that band publishes it
//    (release/acquire at GPU scope), and an export warp copies the band's own
//    last row out for the next band;
//  * matching costs stream into shared memory per row in chunks of
//    kS2CH pixels by bulk asynchronous copies (cp.async.bulk, completion on
//    an mbarrier), kS2NB-1 chunks ahead of the row;
//  * bands are handed out by a ticket counter in dependency order (band b of
//    a sweep after band b-1), so a band only ever waits on bands that some
//    running CTA already owns: no co-residency requirement, any grid size.
//    An exchange row holds a whole image row (no wrap inside a band); band b
//    reuses the exchange row of band b-M after band b-M+1 has imported it.
// Every wait is bounded: on timeout the CTA records LUMEN_ERR_TIMEOUT in
// *status and leaves; CTAs that see a non-zero status stop taking bands.
#pragma once
#include <algorithm>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "sgm_step.cuh"

namespace lumen {

constexpr int kS2Q = 8;     // ring slots between two rows of a band (power of two)
constexpr int kS2CH = 8;    // pixels per cost chunk
constexpr int kS2NB = 3;    // cost chunk buffers per row
constexpr int kS2X = 4;     // pixels per import / export copy step
constexpr int kS2Pub = 4;   // the export publishes its progress every kS2Pub pixels

struct Sweep2Args {
    const uint8_t* cost;     // [H][W][Dp]
    const uint8_t* img;      // [H][W]
    uint16_t* part[2];       // per-sweep partial sums, [H][W][Dp]
    uint8_t* xring;          // [2][M][W][SB] exchange rows
    unsigned* prod;          // [2][nBands] pixels of band b's last row exported
    unsigned* cons;          // [2][nBands] pixels of band b's exchange row imported by band b+1
    unsigned* ticket;        // next band ticket
    int* status;
    int W, H, D, Dp;
    int P1, P2, costScale;
    uint32_t p1x2, bsub;
    int nBands;              // bands per sweep
    int M;                   // exchange rows per sweep (>= 2)
    int QB;                  // slots of the import ring and of the last row's ring (power of two, >= 8)
    long long spinMax;
    int stallTest;           // 1: the first band's first row waits on a counter nothing advances
};

// Shared memory carve-up (bytes), identical on host and device.
struct Sweep2Smem {
    int rings, zero, cost, img, lut, bars, prog, total;
    int Wp, SB;
};
__host__ __device__ inline int sweep2_slot_bytes(int Dp, int NP) { return NP * 2 * Dp + 16; }
__host__ __device__ inline int sweep2_ring_off(int ring, int R, int QB) {
    // ring 0: import (QB slots); ring 1+r: output of row r (kS2Q slots, QB for r = R-1)
    return ring == 0 ? 0 : QB + (ring - 1) * kS2Q;
}
__host__ __device__ inline Sweep2Smem sweep2_smem(int W, int Dp, int R, int NP, int QB) {
    Sweep2Smem s;
    s.Wp = (W + 15) & ~15;
    s.SB = sweep2_slot_bytes(Dp, NP);
    int o = 0;
    s.rings = o;
    o += (2 * QB + (R - 1) * kS2Q) * s.SB;
    s.zero = o;  // an all-zero slot: a path that starts reads it (L' = 0, min L' = 0 gives L = C)
    o += s.SB;
    o = (o + 127) & ~127;
    s.cost = o;
    o += R * kS2NB * kS2CH * Dp;
    s.img = o;
    o += (R + 1) * s.Wp;
    o = (o + 15) & ~15;
    s.lut = o;
    o += 256 * 4;
    s.bars = o;
    o += R * kS2NB * 8;
    s.prog = o;
    o += 16 * 4;
    s.total = o;
    return s;
}

// ---- synchronisation primitives ----
__device__ __forceinline__ unsigned s2_ld_acquire_cta(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.cta.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void s2_st_release_cta(unsigned* p, unsigned v) {
    asm volatile("st.release.cta.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned s2_ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void s2_st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t s2_smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void s2_mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(s2_smem_addr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void s2_bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    const uint32_t b = s2_smem_addr(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            s2_smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(b)
        : "memory");
}
__device__ __forceinline__ bool s2_mbar_try(uint64_t* bar, unsigned parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(s2_smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait until *p >= need (CTA scope).  Returns false (and raises the
// CTA abort flag, recording a timeout) when the wait gives up or another warp
// of the CTA aborted.
// Called by all 32 lanes of a warp; every decision uses lane 0's reads, so the
// warp leaves the wait together.
__device__ __forceinline__ bool s2_wait_cta(const unsigned* p, unsigned need, unsigned& seen,
                                            volatile int* abortFlag, int* status, long long spinMax) {
    unsigned v = __shfl_sync(kFullMask, s2_ld_acquire_cta(p), 0);
    long long k = 0;
    while (v < need) {
        if (__shfl_sync(kFullMask, *abortFlag, 0)) return false;
        if (++k >= spinMax) {
            atomicExch(status, (int)LUMEN_ERR_TIMEOUT);
            *abortFlag = 1;
            return false;
        }
        v = __shfl_sync(kFullMask, s2_ld_acquire_cta(p), 0);
    }
    seen = v;
    return true;
}

// Bounded wait until *p >= need (GPU scope); also gives up when the launch
// has already failed (*status != 0).
// Called by all 32 lanes of a warp (decisions on lane 0's reads, as above).
__device__ __forceinline__ bool s2_wait_gpu(const unsigned* p, unsigned need, volatile int* abortFlag,
                                            int* status, long long spinMax) {
    unsigned v = __shfl_sync(kFullMask, s2_ld_acquire_gpu(p), 0);
    long long k = 0;
    while (v < need) {
        if (__shfl_sync(kFullMask, *abortFlag, 0)) return false;
        if ((k & 255) == 255 && __shfl_sync(kFullMask, *(volatile int*)status, 0) != 0) {
            *abortFlag = 1;
            return false;
        }
        if (++k >= spinMax) {
            atomicExch(status, (int)LUMEN_ERR_TIMEOUT);
            *abortFlag = 1;
            return false;
        }
        v = __shfl_sync(kFullMask, s2_ld_acquire_gpu(p), 0);
    }
    return true;
}

// Copy `bytes` (multiple of 16) with the 32 lanes of a warp: global exchange
// row -> shared memory (loads bypass L1, the row is rewritten between uses) ...
__device__ __forceinline__ void s2_copy_in(void* sdst, const void* gsrc, int bytes, int lane) {
    uint4* d = reinterpret_cast<uint4*>(sdst);
    const uint4* s = reinterpret_cast<const uint4*>(gsrc);
    for (int i = lane; i < bytes / 16; i += 32) d[i] = __ldcg(s + i);
}
// ... and shared memory -> global exchange row.
__device__ __forceinline__ void s2_copy_out(void* gdst, const void* ssrc, int bytes, int lane) {
    uint4* d = reinterpret_cast<uint4*>(gdst);
    const uint4* s = reinterpret_cast<const uint4*>(ssrc);
    for (int i = lane; i < bytes / 16; i += 32) d[i] = s[i];
}

template <int KW, bool WRAP, bool FULL, int NP, int R>
__global__ void __launch_bounds__((R + 2) * 32)
sweep2_kernel(Sweep2Args a) {
    extern __shared__ __align__(128) uint8_t sm[];
    const Sweep2Smem L = sweep2_smem(a.W, a.Dp, R, NP, a.QB);
    uint8_t* rings = sm + L.rings;
    uint8_t* scost = sm + L.cost;
    uint8_t* simg = sm + L.img;
    int* p2lut = reinterpret_cast<int*>(sm + L.lut);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L.bars);
    unsigned* prog = reinterpret_cast<unsigned*>(sm + L.prog);  // [0] import, [1+r] row r, [R+1] export
    volatile int* sflag = reinterpret_cast<volatile int*>(sm + L.prog) + 12;  // [0] ticket, [1] abort

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = a.W, H = a.H, Dp = a.Dp, SB = L.SB, QB = a.QB;
    const int off = lane * 2 * KW;  // first disparity of this lane

    for (int g = threadIdx.x; g < 256; g += blockDim.x) p2lut[g] = max(a.P1 + 1, a.P2 * 8 / max(8, g));
    if (threadIdx.x < R * kS2NB) s2_mbar_init(&bars[threadIdx.x], 1);
    if (threadIdx.x == 0) sflag[1] = 0;
    for (int i = threadIdx.x; i < SB / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sm + L.zero)[i] = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();

    LaneMasks<KW> mk;
    make_lane_masks<KW>(lane, a.D, mk);
    unsigned seq = 0;  // cost chunks this row warp has consumed so far (mbarrier phase)

    for (;;) {
        if (threadIdx.x == 0) {
            int t = (int)atomicAdd(a.ticket, 1u);
            if (*(volatile int*)a.status != 0) t = 2 * a.nBands;
            sflag[0] = t;
        }
        if (threadIdx.x < R + 2) prog[threadIdx.x] = 0;
        __syncthreads();
        const int t = sflag[0];
        if (t >= 2 * a.nBands) break;
        const int sw = t & 1, b = t >> 1;
        const int v0 = b * R;
        const int lastActive = min(R - 1, H - 1 - v0);
        const bool hasPrev = b > 0, hasNext = b + 1 < a.nBands;
        // ---- stage sweep-oriented image rows v0-1 .. v0+R-1 ----
        for (int i = threadIdx.x; i < (R + 1) * W; i += blockDim.x) {
            const int rr = i / W, u = i - rr * W;
            const int vv = v0 - 1 + rr;
            uint8_t val = 0;
            if (vv >= 0 && vv < H) {
                const int x = sw ? W - 1 - u : u, y = sw ? H - 1 - vv : vv;
                val = a.img[(size_t)y * W + x];
            }
            simg[rr * L.Wp + u] = val;
        }
        __syncthreads();

        if (warp == R) {
            // ================= import warp: previous band's last row =================
            if (hasPrev) {
                const uint8_t* src = a.xring + ((size_t)(sw * a.M + (b - 1) % a.M) * W) * SB;
                const unsigned* pprod = a.prod + sw * a.nBands + (b - 1);
                unsigned seen0 = 0;
                bool ok = true;
                for (int p0 = 0; p0 < W && ok; p0 += kS2X) {
                    const int n = min(kS2X, W - p0);
                    ok = s2_wait_gpu(pprod, (unsigned)(p0 + n), sflag + 1, a.status, a.spinMax);
                    const int needRow0 = p0 + kS2X + 1 - QB;  // row 0 done with pixel p - QB + 1
                    if (ok && needRow0 > 0 && seen0 < (unsigned)needRow0)
                        ok = s2_wait_cta(&prog[1], (unsigned)needRow0, seen0, sflag + 1, a.status, a.spinMax);
                    if (!ok) break;
                    s2_copy_in(rings + (size_t)(p0 & (QB - 1)) * SB, src + (size_t)p0 * SB, n * SB, lane);
                    __syncwarp();
                    if (lane == 0) s2_st_release_cta(&prog[0], (unsigned)(p0 + n));
                }
                __syncwarp();
                if (ok && lane == 0) s2_st_release_gpu(a.cons + sw * a.nBands + (b - 1), (unsigned)W);
            }
        } else if (warp == R + 1) {
            // ================= export warp: this band's last row =================
            if (hasNext) {
                uint8_t* dst = a.xring + ((size_t)(sw * a.M + b % a.M) * W) * SB;
                unsigned* oprod = a.prod + sw * a.nBands + b;
                const uint8_t* src = rings + (size_t)sweep2_ring_off(R, R, QB) * SB;
                bool ok = true;
                if (b >= a.M) ok = s2_wait_gpu(a.cons + sw * a.nBands + (b - a.M), (unsigned)W, sflag + 1,
                                               a.status, a.spinMax);
                unsigned seenL = 0;
                for (int p0 = 0; p0 < W && ok; p0 += kS2X) {
                    const int n = min(kS2X, W - p0);
                    if (seenL < (unsigned)(p0 + n))
                        ok = s2_wait_cta(&prog[R], (unsigned)(p0 + n), seenL, sflag + 1, a.status, a.spinMax);
                    if (!ok) break;
                    s2_copy_out(dst + (size_t)p0 * SB, src + (size_t)(p0 & (QB - 1)) * SB, n * SB, lane);
                    __syncwarp();
                    if (lane == 0) s2_st_release_cta(&prog[R + 1], (unsigned)(p0 + n));
                    if (((p0 + n) % kS2Pub) == 0 || p0 + n == W) {
                        __threadfence();
                        __syncwarp();
                        if (lane == 0) s2_st_release_gpu(oprod, (unsigned)(p0 + n));
                    }
                }
            }
        } else if (warp <= lastActive) {
            // ================= row warp =================
            const int r = warp;
            const int v = v0 + r;
            const int y = sw ? H - 1 - v : v;
            const bool startV = (v == 0);
            const bool isLast = (r == lastActive);
            const bool writes = !isLast || hasNext;  // someone reads this row's ring
            const uint8_t* pring = rings + (size_t)sweep2_ring_off(r, R, QB) * SB;
            const int pQm = (r == 0 ? QB : kS2Q) - 1;
            uint8_t* oring = rings + (size_t)sweep2_ring_off(r + 1, R, QB) * SB;
            const int oQ = (r == R - 1) ? QB : kS2Q;
            const uint8_t* zslot = sm + L.zero;
            const unsigned* predProg = &prog[r];
            unsigned* myProg = &prog[r + 1];
            const unsigned* succProg = &prog[r + 2];
            const uint8_t* crow = a.cost + (size_t)y * W * Dp;
            // partial-volume pointer of pixel u = 0 (this lane's words), stepping by +-Dp
            uint16_t* pout = (sw ? a.part[1] : a.part[0]) + ((size_t)y * W + (sw ? W - 1 : 0)) * Dp + off;
            const ptrdiff_t pstep = sw ? -(ptrdiff_t)Dp : (ptrdiff_t)Dp;
            uint8_t* cbase = scost + (size_t)r * kS2NB * kS2CH * Dp;
            uint64_t* rbars = bars + r * kS2NB;
            const uint8_t* irow = simg + (r + 1) * L.Wp;
            const uint8_t* iprev = simg + r * L.Wp;
            const int nCh = (W + kS2CH - 1) / kS2CH;

            auto issue = [&](int c) {
                const int n = min(kS2CH, W - c * kS2CH);
                const int xlo = sw ? W - (c * kS2CH + n) : c * kS2CH;
                const unsigned slot = (seq + (unsigned)c) % kS2NB;
                s2_bulk_load(cbase + (size_t)slot * kS2CH * Dp, crow + (size_t)xlo * Dp, (unsigned)(n * Dp),
                             &rbars[slot]);
            };
            if (lane == 0)
                for (int c = 0; c < kS2NB - 1 && c < nCh; ++c) issue(c);
            int issued = min(kS2NB - 1, nCh);

            // L' = 0 and min L' = 0 before pixel 0: the first step yields L = C
            uint32_t LH[KW];
#pragma unroll
            for (int w = 0; w < KW; ++w) LH[w] = 0;
            uint32_t minH = 0;
            uint32_t p2HV = 0, p2D = 0;  // adaptive P2 of pixel u0 + lane: (H | V << 16), (D1 | D2 << 16)
            unsigned seenPred = startV ? (unsigned)W : 0u, seenSucc = 0;
            bool ok = true;
            if (a.stallTest && t == 0 && r == 0) {
                // failure-path self test: the export never reaches pixel W + 1, so this
                // bounded wait runs out and the launch ends with LUMEN_ERR_TIMEOUT
                unsigned never = 0;
                ok = s2_wait_cta(&prog[R + 1], (unsigned)W + 1u, never, sflag + 1, a.status, a.spinMax);
            }
            int c = 0;
            for (; c < nCh && ok; ++c) {
                if (c + kS2NB - 1 < nCh) {
                    if (lane == 0) issue(c + kS2NB - 1);
                    ++issued;
                }
                const int u0 = c * kS2CH;
                if ((u0 & 31) == 0) {
                    // adaptive P2 (src/sgbm_kernels.cu:301-310) of the next 32 pixels, one per lane
                    const int pu = u0 + lane;
                    uint32_t hv = 0, dd = 0;
                    if (pu < W) {
                        const int cur = irow[pu];
                        const uint32_t ph = (uint32_t)p2lut[abs(cur - irow[max(pu - 1, 0)])] & 0xFFFFu;
                        const uint32_t pv = (uint32_t)p2lut[abs(cur - iprev[pu])] & 0xFFFFu;
                        hv = ph | (pv << 16);
                        if (NP == 3) {
                            const uint32_t p1 = (uint32_t)p2lut[abs(cur - iprev[max(pu - 1, 0)])] & 0xFFFFu;
                            const uint32_t p3 = (uint32_t)p2lut[abs(cur - iprev[min(pu + 1, W - 1)])] & 0xFFFFu;
                            dd = p1 | (p3 << 16);
                        }
                    }
                    p2HV = hv;
                    p2D = dd;
                }
                {
                    const unsigned slot = (seq + (unsigned)c) % kS2NB;
                    const unsigned parity = ((seq + (unsigned)c) / kS2NB) & 1u;
                    long long k = 0;
                    while (!__shfl_sync(kFullMask, (int)s2_mbar_try(&rbars[slot], parity), 0)) {
                        if (++k >= a.spinMax || __shfl_sync(kFullMask, sflag[1], 0)) {
                            if (k >= a.spinMax) { atomicExch(a.status, (int)LUMEN_ERR_TIMEOUT); sflag[1] = 1; }
                            ok = false;
                            break;
                        }
                    }
                    if (!ok) break;
                }
                const uint8_t* cbuf = cbase + (size_t)((seq + (unsigned)c) % kS2NB) * kS2CH * Dp;
                const int n = min(kS2CH, W - u0);
                for (int j = 0; j < n; ++j) {
                    const int u = u0 + j;
                    // ---- wait for the predecessor's pixels u-1 .. u+1 and a free output slot ----
                    const unsigned need = (unsigned)min(u + (NP == 3 ? 2 : 1), W);
                    if (seenPred < need &&
                        !s2_wait_cta(predProg, need, seenPred, sflag + 1, a.status, a.spinMax)) { ok = false; break; }
                    const int needS = u - oQ + 2;
                    if (writes && needS > 0 && seenSucc < (unsigned)needS &&
                        !s2_wait_cta(succProg, (unsigned)needS, seenSucc, sflag + 1, a.status, a.spinMax)) { ok = false; break; }
                    // ---- inputs ----
                    const int jj = sw ? n - 1 - j : j;
                    uint32_t Cw[KW];
                    load_cost_words<KW>(cbuf + (size_t)jj * Dp + off, Cw);
#pragma unroll
                    for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(Cw[w], a.costScale);
                    const uint32_t hv = __shfl_sync(kFullMask, p2HV, u & 31);
                    const uint32_t dd = NP == 3 ? __shfl_sync(kFullMask, p2D, u & 31) : 0u;
                    uint32_t Lp[NP][KW], Ln[NP][KW], mp[NP], LnH[KW];
                    int p2v[NP];
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth) {
                        // path start (first sweep row, or the neighbour left / right of the
                        // image): read the zero slot
                        const uint8_t* slot;
                        if (pth == 0) slot = startV ? zslot : pring + (size_t)(u & pQm) * SB;
                        else if (pth == 1) slot = (startV || u == 0) ? zslot : pring + (size_t)((u - 1) & pQm) * SB;
                        else slot = (startV || u == W - 1) ? zslot : pring + (size_t)((u + 1) & pQm) * SB;
                        load_words<KW>(reinterpret_cast<const uint16_t*>(slot + pth * 2 * Dp) + off, Lp[pth]);
                        mp[pth] = reinterpret_cast<const uint32_t*>(slot + NP * 2 * Dp)[pth];
                        p2v[pth] = pth == 0 ? (int)(hv >> 16) : (pth == 1 ? (int)(dd & 0xFFFFu) : (int)(dd >> 16));
                    }
                    // ---- recurrences: H, then V (u), D1 (u-1), D2 (u+1) ----
                    sgm_step<KW, WRAP, FULL, 32>(LH, Cw, minH, (int)(hv & 0xFFFFu), a.p1x2, a.bsub, mk, LnH);
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth)
                        sgm_step<KW, WRAP, FULL, 32>(Lp[pth], Cw, mp[pth], p2v[pth], a.p1x2, a.bsub, mk, Ln[pth]);
                    minH = warp_min_u16<KW, 32>(LnH);
                    uint32_t mn[NP];
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth) mn[pth] = warp_min_u16<KW, 32>(Ln[pth]);
                    uint32_t S[KW];
#pragma unroll
                    for (int w = 0; w < KW; ++w) {
                        LH[w] = LnH[w];
                        S[w] = LnH[w];
                    }
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth)
#pragma unroll
                        for (int w = 0; w < KW; ++w) S[w] = WRAP ? __vadd2(S[w], Ln[pth][w]) : S[w] + Ln[pth][w];
                    // ---- outputs ----
                    if (writes) {
                        uint8_t* slot = oring + (size_t)(u & (oQ - 1)) * SB;
#pragma unroll
                        for (int pth = 0; pth < NP; ++pth)
                            store_words<KW>(reinterpret_cast<uint16_t*>(slot + pth * 2 * Dp) + off, Ln[pth]);
                        if (lane == 0) {
                            if (NP == 3)
                                *reinterpret_cast<uint4*>(slot + NP * 2 * Dp) = make_uint4(mn[0], mn[NP > 1 ? 1 : 0], mn[NP > 2 ? 2 : 0], 0u);
                            else
                                *reinterpret_cast<uint32_t*>(slot + NP * 2 * Dp) = mn[0];
                        }
                    }
                    store_words<KW>(pout, S);
                    pout += pstep;
                    __syncwarp();
                    if (lane == 0) s2_st_release_cta(myProg, (unsigned)(u + 1));
                }
            }
            // drain bulk copies still in flight (only after an abort)
            for (int cc = c; cc < issued; ++cc) {
                const unsigned slot = (seq + (unsigned)cc) % kS2NB;
                const unsigned parity = ((seq + (unsigned)cc) / kS2NB) & 1u;
                long long k = 0;
                while (!__shfl_sync(kFullMask, (int)s2_mbar_try(&rbars[slot], parity), 0) && ++k < a.spinMax) {
                }
            }
            seq += (unsigned)issued;
        }
        __syncthreads();
        if (sflag[1]) break;
    }
}

}  // namespace lumen
