// sweep_kernel.cuh -- SGM aggregation as two fused wavefront sweeps (schedule 2).
//
// The eight path recurrences of the reference (src/sgbm_kernels.cu:315-742)
// are regrouped by the neighbour they read:
//   forward sweep  F: LR (x-1,y)  TB (x,y-1)  TLBR (x-1,y-1)  TRBL (x+1,y-1)
//   backward sweep B: RL (x+1,y)  BT (x,y+1)  BRTL (x+1,y+1)  BLTR (x-1,y+1)
// B is F with the image mirrored in both axes, so one kernel body runs both in
// "sweep coordinates" (u, v): x = u or W-1-u, y = v or H-1-v.  A pixel needs
// its own row's previous pixel and the previous row's pixels u-1, u, u+1, so
// rows advance as a wavefront with row v+1 two pixels behind row v.
//
// Work decomposition: a CTA owns a band of R consecutive sweep rows and walks
// them in lockstep (one __syncthreads per step), teams of T lanes per row
// (T = 32, 16 or 8; lane holds 2*KW disparities, sgm_step.cuh).  Row r hands
// its TB/TLBR/TRBL vectors to row r+1 through a 4-slot shared-memory ring; the
// band's last row hands them to the next band (another CTA) through a global
// ring with release/acquire progress counters, and the next band prefetches
// them with cp.async.  Cost vectors are prefetched the same way.  The four
// path vectors of a pixel are summed in registers and stored once: each sweep
// writes one uint16 partial volume, no read-modify-write of the aggregate.
//
// All CTAs are co-resident (cooperative launch); a CTA that runs out of bands
// exits.  Every wait is a bounded spin: on timeout the CTA records
// LUMEN_ERR_TIMEOUT in *status and leaves its band (all its warps together).
#pragma once
#include <algorithm>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"
#include "sgm_step.cuh"

namespace lumen {

constexpr int kLag = 4;        // prefetch distance (steps) of cost / exchange copies
constexpr int kRowSlots = 4;   // smem ring slots per band row
constexpr int kXSlots = 8;     // smem ring slots of the incoming (previous band's) row
constexpr int kCostSlots = 8;  // smem cost slots per row
constexpr int kPublish = 4;    // publish progress every kPublish steps

struct SweepArgs {
    const uint8_t* cost;
    const uint8_t* img;
    uint16_t* part[2];       // per-sweep partial sums, [H][W][Dp]
    uint8_t* xring;          // [2][G][W][3][slotBytes]
    unsigned* prod;          // [2][G] pixels published (monotonic over the launch)
    unsigned* cons;          // [2][G] pixels consumed
    int* status;
    int W, H, D, Dp;
    int P1, P2, costScale;
    uint32_t p1x2, bsub;
    int R;                   // rows per band
    int nBands;              // per sweep
    int G;                   // CTAs per sweep
    int slotBytes;           // 2*Dp + 16
    int K;                   // exchange ring capacity in pixels (W, or fewer when one wave)
    long long spinMax;
    int plan;                // 1: only compute the grid (G) into *gridOut, launch nothing
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Shared memory carve-up (bytes), identical on host and device.
struct SweepSmem {
    int imgOff, ringOff, xOff, costOff, lutOff, total;
    int Wp, slotBytes;
};
__host__ __device__ inline SweepSmem sweep_smem(int W, int Dp, int R) {
    SweepSmem s;
    s.Wp = (W + 15) & ~15;
    s.slotBytes = 2 * Dp + 16;
    s.imgOff = 0;
    int o = (R + 1) * s.Wp;
    o = (o + 15) & ~15;
    s.ringOff = o;
    o += R * 3 * kRowSlots * s.slotBytes;
    s.xOff = o;
    o += 3 * kXSlots * s.slotBytes;
    s.costOff = o;
    o += R * kCostSlots * Dp;
    s.lutOff = o;
    o += 256 * 4;
    s.total = o;
    return s;
}

template <int T, int KW, bool WRAP, bool FULL, int NW, int NP>
__global__ void __launch_bounds__(NW * 32)
sweep_kernel(SweepArgs a) {
    constexpr int RPW = 32 / T;  // rows per warp
    extern __shared__ __align__(16) uint8_t sm[];
    const SweepSmem L = sweep_smem(a.W, a.Dp, a.R);
    uint8_t* simg = sm + L.imgOff;
    uint8_t* sring = sm + L.ringOff;
    uint8_t* sx = sm + L.xOff;
    uint8_t* scost = sm + L.costOff;
    int* p2lut = reinterpret_cast<int*>(sm + L.lutOff);
    __shared__ int abortFlag;

    const int sw = blockIdx.x & 1;   // 0 forward, 1 backward
    const int c = blockIdx.x >> 1;   // CTA index within the sweep
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = lane / T, tl = lane & (T - 1);
    const int r = warp * RPW + team;  // band row of this team
    const int W = a.W, H = a.H, Dp = a.Dp;
    const int off = tl * 2 * KW;      // first disparity of this lane
    const int SB = L.slotBytes;

    for (int g = threadIdx.x; g < 256; g += blockDim.x)
        p2lut[g] = max(a.P1 + 1, a.P2 * 8 / max(8, g));
    if (threadIdx.x == 0) abortFlag = 0;

    LaneMasks<KW> mk;
    make_lane_masks<KW>(tl, a.D, mk);
    uint16_t* part = sw ? a.part[1] : a.part[0];
    const size_t ringStride = (size_t)a.K * 3 * SB;

    for (int b = c; b < a.nBands; b += a.G) {
        const int it = b / a.G;
        const int v0 = b * a.R;
        const int v = v0 + r;
        const bool rowOk = r < a.R && v < H;
        // ---- stage sweep-oriented image rows v0-1 .. v0+R-1 ----
        __syncthreads();
        for (int i = threadIdx.x; i < (a.R + 1) * W; i += blockDim.x) {
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
        // incoming ring of the previous band (produced by CTA (b-1) % G, iteration (b-1) / G)
        const bool hasPrev = b > 0;
        const int pc = (b - 1 + a.G) % a.G;
        const unsigned pBase = hasPrev ? (unsigned)((b - 1) / a.G) * (unsigned)W : 0u;
        const uint8_t* pring = a.xring + ((size_t)sw * a.G + pc) * ringStride;
        unsigned* pProd = a.prod + sw * a.G + pc;
        unsigned* pCons = a.cons + sw * a.G + pc;
        // outgoing ring (this CTA, iteration it)
        const bool hasNext = b + 1 < a.nBands;
        uint8_t* oring = a.xring + ((size_t)sw * a.G + c) * ringStride;
        unsigned* oProd = a.prod + sw * a.G + c;
        unsigned* oCons = a.cons + sw * a.G + c;
        const unsigned oBase = (unsigned)it * (unsigned)W;
        unsigned seenProd = 0, seenCons = 0;
        const bool lastRow = (r == a.R - 1) || (v == H - 1);
        const bool firstRow = (r == 0);

        uint32_t LH[KW];
#pragma unroll
        for (int w = 0; w < KW; ++w) LH[w] = 0;
        uint32_t minH = 0;
        const int sEnd = W - 1 + 2 * (a.R - 1);
        for (int s = -kLag - 1; s <= sEnd; ++s) {
            const int u = s - 2 * r;
            // ---- prefetch: cost of pixel u+kLag for this row ----
            {
                const int pu = u + kLag;
                if (rowOk && pu >= 0 && pu < W) {
                    const int x = sw ? W - 1 - pu : pu, y = sw ? H - 1 - v : v;
                    const uint8_t* src = a.cost + ((size_t)y * W + x) * Dp;
                    uint8_t* dst = scost + (r * kCostSlots + (pu & (kCostSlots - 1))) * Dp;
                    for (int k = tl; k < Dp / 16; k += T) cp_async16(dst + 16 * k, src + 16 * k);
                }
            }
            // ---- prefetch: previous band's row, pixel s+kLag+1 (warp 0) ----
            if (warp == 0 && hasPrev) {
                const int pu = s + kLag + 1;
                if (pu >= 0 && pu < W) {
                    const unsigned need = pBase + (unsigned)pu + 1u;
                    if (seenProd < need) {
                        long long spins = 0;
                        unsigned pv = ld_acquire(pProd);
                        while (pv < need && ++spins < a.spinMax) pv = ld_acquire(pProd);
                        if (pv < need) {
                            if (lane == 0) { atomicExch(a.status, (int)LUMEN_ERR_TIMEOUT); abortFlag = 1; }
                            pv = need;  // leave the loop; abortFlag stops the band below
                        }
                        seenProd = pv;
                    }
                    const uint8_t* src = pring + (size_t)((pBase + (unsigned)pu) % (unsigned)a.K) * 3 * SB;
                    uint8_t* dst = sx + (pu & (kXSlots - 1)) * 3 * SB;
                    for (int k = lane; k < 3 * SB / 16; k += 32) cp_async16(dst + 16 * k, src + 16 * k);
                }
            }
            cp_async_commit();

            // ---- back-pressure: the outgoing slot of pixel u was last used one
            //      iteration ago; wait until that pixel was consumed ----
            const bool active = rowOk && u >= 0 && u < W;
            const unsigned teamMask = T == 32 ? 0xFFFFFFFFu : (((1u << T) - 1u) << (team * T));
            if (hasNext && active && lastRow && oBase + (unsigned)u >= (unsigned)a.K) {
                const unsigned need = oBase + (unsigned)u + 1u - (unsigned)a.K;
                if (seenCons < need) {
                    unsigned cv = 0;
                    if (tl == 0) {
                        long long spins = 0;
                        cv = ld_acquire(oCons);
                        while (cv < need && ++spins < a.spinMax) cv = ld_acquire(oCons);
                        if (cv < need) { atomicExch(a.status, (int)LUMEN_ERR_TIMEOUT); abortFlag = 1; cv = need; }
                    }
                    seenCons = __shfl_sync(teamMask, cv, 0, T);
                }
            }
            // ---- compute pixel u of row r: every lane of the warp runs the math
            //      (teams of one warp sit at different u), stores are predicated.
            //      All inputs are loaded first and the NP+1 recurrences are
            //      independent, so their shuffles and reductions overlap. ----
            {
                const int uc = min(max(u, 0), W - 1);
                const int x = sw ? W - 1 - uc : uc, y = sw ? H - 1 - min(v, H - 1) : min(v, H - 1);
                uint32_t Cw[KW], S[KW], LnH[KW];
                uint32_t Lp[NP][KW], Ln[NP][KW], mp[NP];
                int p2v[NP];
                load_cost_words<KW>(scost + (r * kCostSlots + (uc & (kCostSlots - 1))) * Dp + off, Cw);
#pragma unroll
                for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(Cw[w], a.costScale);
                const uint8_t* irow = simg + (r + 1) * L.Wp;
                const uint8_t* iprev = simg + r * L.Wp;
                const int cur = irow[uc];
                const int p2h = p2lut[abs(cur - irow[max(uc - 1, 0)])];
#pragma unroll
                for (int pth = 0; pth < NP; ++pth) {
                    const int pu = pth == 0 ? uc : (pth == 1 ? uc - 1 : uc + 1);
                    const int puc = min(max(pu, 0), W - 1);
                    // firstRow reads the previous band's row, other rows row r-1
                    // (row 0 of band 0 starts every path: its slot is not used)
                    const uint8_t* slot;
                    if (firstRow) slot = sx + ((puc & (kXSlots - 1)) * 3 + pth) * SB;
                    else slot = sring + ((max(r - 1, 0) * 3 + pth) * kRowSlots + (puc & (kRowSlots - 1))) * SB;
                    load_words<KW>(reinterpret_cast<const uint16_t*>(slot) + off, Lp[pth]);
                    mp[pth] = *reinterpret_cast<const uint32_t*>(slot + 2 * Dp) & 0xFFFFu;
                    p2v[pth] = p2lut[abs(cur - iprev[puc])];
                }
                // H path (LR / RL) and the vertical-ish paths: 0 = V (u), 1 = D1 (u-1),
                // 2 = D2 (u+1); NP = 1 (4-path mode) runs V only.  A path start
                // selects C instead of the step's result.
                sgm_step<KW, WRAP, FULL, T>(LH, Cw, minH, p2h, a.p1x2, a.bsub, mk, LnH);
#pragma unroll
                for (int pth = 0; pth < NP; ++pth)
                    sgm_step<KW, WRAP, FULL, T>(Lp[pth], Cw, mp[pth], p2v[pth], a.p1x2, a.bsub, mk, Ln[pth]);
                if (uc == 0) {
#pragma unroll
                    for (int w = 0; w < KW; ++w) LnH[w] = Cw[w] | mk.padMask[w];
                }
#pragma unroll
                for (int pth = 0; pth < NP; ++pth) {
                    const int pu = pth == 0 ? uc : (pth == 1 ? uc - 1 : uc + 1);
                    if ((v == 0) || pu < 0 || pu >= W) {
#pragma unroll
                        for (int w = 0; w < KW; ++w) Ln[pth][w] = Cw[w] | mk.padMask[w];
                    }
                }
                const uint32_t mnH = warp_min_u16<KW, T>(LnH);
                uint32_t mn[NP];
#pragma unroll
                for (int pth = 0; pth < NP; ++pth) mn[pth] = warp_min_u16<KW, T>(Ln[pth]);
                if (active) {
#pragma unroll
                    for (int w = 0; w < KW; ++w) LH[w] = LnH[w];
                    minH = mnH;
                }
#pragma unroll
                for (int w = 0; w < KW; ++w) S[w] = LnH[w];
#pragma unroll
                for (int pth = 0; pth < NP; ++pth)
#pragma unroll
                    for (int w = 0; w < KW; ++w) S[w] = WRAP ? __vadd2(S[w], Ln[pth][w]) : S[w] + Ln[pth][w];
                if (active) {
                    uint8_t* outSlot = sring + ((r * 3) * kRowSlots + (uc & (kRowSlots - 1))) * SB;
                    uint8_t* xout = oring + ((size_t)((oBase + (unsigned)uc) % (unsigned)a.K) * 3) * SB;
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth) {
                        uint8_t* myslot = outSlot + pth * kRowSlots * SB;
                        store_words<KW>(reinterpret_cast<uint16_t*>(myslot) + off, Ln[pth]);
                        if (tl == 0) *reinterpret_cast<uint32_t*>(myslot + 2 * Dp) = mn[pth];
                        if (lastRow && hasNext) {
                            uint8_t* xs = xout + pth * SB;
                            store_words<KW>(reinterpret_cast<uint16_t*>(xs) + off, Ln[pth]);
                            if (tl == 0) *reinterpret_cast<uint32_t*>(xs + 2 * Dp) = mn[pth];
                        }
                    }
                    store_words<KW>(part + ((size_t)y * W + x) * Dp + off, S);
                }
            }
            // ---- publish the band's last row to the next band ----
            if (hasNext && active && lastRow && ((u % kPublish) == kPublish - 1 || u == W - 1)) {
                __threadfence();
                __syncwarp(teamMask);
                if (tl == 0) st_release(oProd, oBase + (unsigned)u + 1u);
            }
            cp_async_wait<kLag - 1>();
            __syncthreads();
            // ---- consumer progress (copies of pixel s-kLag+1+kLag+1 = s+2 are complete) ----
            if (warp == 0 && lane == 0 && hasPrev) {
                const int done = s + 2;  // exchange pixels < done are in shared memory
                if (done > 0 && ((done % kPublish) == 0 || done >= W)) st_release(pCons, pBase + (unsigned)min(done, W));
            }
            if (abortFlag) break;
        }
        cp_async_wait<0>();
        __syncthreads();
        if (abortFlag) return;
    }
}

// ---------------------------------------------------------------------------
// launch helpers (instantiated per configuration in sweep_cfg_*.cu)
// ---------------------------------------------------------------------------
template <int T, int KW, bool WRAP, bool FULL, int NW, int NP>
cudaError_t sweep_launch_t(SweepArgs a, cudaStream_t s, int numSMs, int* gridOut) {
    auto kern = sweep_kernel<T, KW, WRAP, FULL, NW, NP>;
    const SweepSmem L = sweep_smem(a.W, a.Dp, a.R);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
    if (e != cudaSuccess) return e;
    int perSM = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, NW * 32, L.total);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    const int maxG = perSM * numSMs / 2;
    a.G = std::min(a.nBands, maxG);
    if (a.G < 1) return cudaErrorInvalidConfiguration;
    *gridOut = a.G;
    if (a.plan) return cudaSuccess;
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)kern, dim3(2 * a.G), dim3(NW * 32), args,
                                       (size_t)L.total, s);
}

// Lanes per pixel T and words per lane KW = Dp/(2T); NW warps per CTA.
// WRAP (modular uint16 arithmetic) is instantiated for the T = 32, NW = 4
// configurations only; the others serve the no-wrap parameter range.
template <int T, int KW, int NW, int NP>
cudaError_t sweep_launch_np(SweepArgs a, bool wrap, cudaStream_t s, int numSMs, int* g) {
    const bool full = (a.D == a.Dp);
    if constexpr (T == 32 && NW == 4) {
        if (wrap) return full ? sweep_launch_t<T, KW, true, true, NW, NP>(a, s, numSMs, g)
                              : sweep_launch_t<T, KW, true, false, NW, NP>(a, s, numSMs, g);
    } else {
        if (wrap) return cudaErrorInvalidValue;
    }
    return full ? sweep_launch_t<T, KW, false, true, NW, NP>(a, s, numSMs, g)
                : sweep_launch_t<T, KW, false, false, NW, NP>(a, s, numSMs, g);
}

}  // namespace lumen
