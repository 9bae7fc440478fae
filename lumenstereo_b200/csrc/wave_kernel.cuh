// wave_kernel.cuh -- SGM aggregation as two fused wavefront sweeps run by
// lockstep row bands (schedule 4).
//
// Same regrouping of the reference's eight path kernels
// (src/sgbm_kernels.cu:315-742) as the other fused schedules:
//   forward sweep  F: LR (x-1,y)  TB (x,y-1)  TLBR (x-1,y-1)  TRBL (x+1,y-1)
//   backward sweep B: RL (x+1,y)  BT (x,y+1)  BRTL (x+1,y+1)  BLTR (x-1,y+1)
// in sweep coordinates (u, v): x = u or W-1-u, y = v or H-1-v.  The path
// vectors of a pixel are summed in registers and stored once per sweep (one
// uint16 partial volume per sweep).
//
// Work decomposition:
//  * a CTA owns a band of R consecutive sweep rows, one warp per row (a lane
//    holds 2*KW disparities as KW packed uint16x2 words).  The wavefront is
//    latency-bound (its span is about W + 2H steps), so a row keeps all 32
//    lanes: narrower lane teams cut instructions per pixel but lengthen the
//    dependent chain of a step, and redux.sync on a partial mask is slow;
//  * all row warps advance in lockstep, one named barrier (rows only) per
//    step: at step t row r handles pixel u = t - LAG*r (LAG = 2 with the
//    diagonal paths, 1 without), so everything row r needs from row r-1
//    (pixels u-1, u, u+1) was produced in an earlier step and sits in a
//    4-slot shared-memory ring;
//  * matching costs are prefetched per step with cp.async, kWPF-1 pixels
//    ahead, into a per-row ring; adaptive P2 is looked up per pixel from the
//    staged image rows;
//  * an import warp and an export warp, outside the row barrier, move the
//    band's first input row and last output row through a kWK-pixel exchange
//    ring per band boundary in global memory (L2-resident): the export warp
//    publishes progress every kWE pixels (release at GPU scope) and never
//    overwrites a slot the next band has not copied yet; the import warp
//    copies slots (cp.async) as soon as they are published.  They talk to rows
//    0 and R-1 through shared-memory counters (acquire/release at CTA scope),
//    so global-memory latency never stalls a step;
//  * bands are handed out by a ticket counter in dependency order (band b of a
//    sweep after band b-1), and a CTA takes a ticket only while it runs.  A
//    band waits on the band above it (its input) and, through the exchange
//    ring's back-pressure, on the next wave_lookahead_bands(W) bands below it;
//    all of those tickets lie within a window after its own, so a grid of
//    window + 1 resident CTAs always lets the oldest unfinished band finish.
// Every wait is bounded: on timeout the CTA records LUMEN_ERR_TIMEOUT in
// *status and stops; CTAs that see a non-zero status stop taking bands.
//
// Recurrence (src/sgbm_kernels.cu:338-360): packed uint16x2 words.  The
// no-wrap mode takes one three-input minimum and one add-minimum (the DPX
// forms __vimin3_u16x2, __viaddmin_u16x2; measured at half the issue rate of
// __vminu2 on B200, lumen_debug_op_rates) and L = m + C - minL' as one IADD3;
// the wrap mode keeps per-halfword modular adds and two-input minima.  A
// lane's words are reduced with three-input minima; the warp minimum comes
// back from redux.sync (full-warp rows) or an xor butterfly (lane teams).
#pragma once
#include <algorithm>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "sgm_step.cuh"

namespace lumen {

constexpr int kWQ = 4;     // ring slots between consecutive rows of a band
constexpr int kWPF = 8;    // per-row cost ring (pixels); kWPF-1 prefetched ahead
constexpr int kWK = 256;   // global exchange ring per band boundary (pixels, power of two)
constexpr int kWE = 4;     // export progress published every kWE pixels
// Import / export ring slots (QI, QX) are powers of two chosen by the host to
// fit shared memory: 16 or 8.  The import warp keeps two pixel copies in
// flight: a deeper pipeline adds lag to every band hand-off, which costs more
// than it hides.

// One stereo pair of a launch: its volumes, exchange rings and parameters.
struct WaveJob {
    const uint8_t* cost;     // [H][W][Dp]
    const uint8_t* img;      // [H][W] left gray image (adaptive P2)
    uint16_t* part[2];       // per-sweep partial sums, [H][W][Dp]
    uint8_t* xring;          // [2][nBands][kWK][SB] exchange rings
    unsigned* prod;          // [2][nBands] pixels band b has exported
    unsigned* cons;          // [2][nBands] pixels of band b's ring band b+1 has copied
    int W, H, D, nBands;     // nBands: bands per sweep
    int P1, P2, costScale;
    uint32_t p1x2, bsub;
};

// A launch: one pair (`job`, tickets t -> sweep t & 1, band t >> 1) or a batch
// of pairs of one kernel class (`jobs`, tickets through `table`, each entry
// pair << 20 | sweep << 19 | band, every band listed after the band before it
// in its own sweep).
struct WaveArgs {
    WaveJob job;             // the pair when jobs == nullptr
    const WaveJob* jobs;     // batch: [pairs]
    const uint32_t* table;   // batch: [nTickets]
    int nTickets;
    int Wmax;                // widest image (shared-memory carve-up)
    unsigned* ticket;        // next ticket
    int* status;
    int Dp;
    int QI, QX;              // import / export ring slots (16 or 8)
    long long spinMax;
    int stallTest;           // 1: ticket 2 (a band with a predecessor) waits on a pixel never exported
    unsigned long long* trace;  // optional [nTickets][4] band timeline
};

// Band timeline record (diagnostics, lumen_sgbm_debug_trace): per band ticket
// 2 * band + sweep, [0] globaltimer ns when the band's first row finished the
// middle pixel (u = W / 2), [1] when its last row did, [2] when the band
// ended, [3] SM id << 48 | import polls << 32 | export polls << 16 | row waits
// on the helpers (saturating 16-bit counts).  Consecutive bands' [0] give the
// stagger, [0] of band b+1 minus [1] of band b the hand-off.
__device__ __forceinline__ unsigned long long wave_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Shared memory carve-up (bytes), identical on host and device.
struct WaveSmem {
    int rings, imp, exp, zero, cost, img, lut, misc, total;
    int Wp, SB;
};
__host__ __device__ constexpr int wave_slot_bytes(int Dp, int NP) { return NP * 2 * Dp + 16; }
__host__ __device__ inline WaveSmem wave_smem(int W, int Dp, int R, int NP, int QI, int QX) {
    WaveSmem s;
    s.Wp = (W + 15) & ~15;
    s.SB = wave_slot_bytes(Dp, NP);
    int o = 0;
    s.rings = o;
    o += (R - 1) * kWQ * s.SB;
    s.imp = o;
    o += QI * s.SB;
    s.exp = o;
    o += QX * s.SB;
    s.zero = o;  // all-zero slot: a path that starts reads it (L' = 0, min L' = 0 gives L = C)
    o += s.SB;
    o = (o + 127) & ~127;
    s.cost = o;
    o += R * kWPF * Dp;
    s.img = o;
    o += (R + 1) * s.Wp;
    o = (o + 15) & ~15;
    s.lut = o;
    o += 256 * 4;
    s.misc = o;
    o += 32 * 4;
    s.total = o;
    return s;
}

// ---- synchronisation primitives ----
__device__ __forceinline__ unsigned w_ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void w_st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t w_smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned w_ld_acquire_cta(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];\n" : "=r"(v) : "r"(w_smem_addr(p)) : "memory");
    return v;
}
__device__ __forceinline__ void w_st_release_cta(unsigned* p, unsigned v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;\n" ::"r"(w_smem_addr(p)), "r"(v) : "memory");
}
// Named barrier 1 over the band's row-warp threads.
__device__ __forceinline__ void w_rows_barrier(int nThreads) {
    asm volatile("bar.sync 1, %0;\n" ::"r"(nThreads) : "memory");
}
__device__ __forceinline__ void w_cp_async16(uint32_t smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem), "l"(gmem) : "memory");
}
__device__ __forceinline__ void w_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void w_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bounded wait (whole warp) until *p >= need, GPU scope.  `cache` keeps the
// last value seen so satisfied waits cost no load.  Returns false (after
// raising the CTA abort flag) on timeout, on another warp's abort, or when
// the launch has already failed (*status != 0).
__device__ __forceinline__ bool w_wait_gpu(const unsigned* p, unsigned need, unsigned& cache,
                                           volatile int* abortFlag, int* status, long long spinMax,
                                           int lane, volatile int* polls = nullptr) {
    if (cache >= need) return true;
    if (polls && lane == 0) atomicAdd((int*)polls, 1);
    long long k = 0;
    for (;;) {
        unsigned v = 0;
        if (lane == 0) v = w_ld_acquire_gpu(p);
        v = __shfl_sync(kFullMask, v, 0);
        if (v >= need) {
            __syncwarp();
            cache = v;
            return true;
        }
        if (__shfl_sync(kFullMask, *abortFlag, 0)) return false;
        if ((k & 63) == 63 && __shfl_sync(kFullMask, *(volatile int*)status, 0) != 0) {
            *abortFlag = 1;
            return false;
        }
        if (++k >= spinMax) {
            if (lane == 0) atomicExch(status, (int)LUMEN_ERR_TIMEOUT);
            *abortFlag = 1;
            return false;
        }
        __nanosleep(32);
    }
}

// Bounded wait (whole warp) until the shared counter *p >= need (CTA scope;
// every lane acquires its own sufficient value).
__device__ __forceinline__ bool w_wait_cta(const unsigned* p, unsigned need, unsigned& cache,
                                           volatile int* abortFlag, int* status, long long spinMax,
                                           volatile int* polls = nullptr) {
    if (cache >= need) return true;
    unsigned v = w_ld_acquire_cta(p);
    if (__all_sync(kFullMask, v >= need)) {
        cache = __shfl_sync(kFullMask, v, 0);
        return true;
    }
    if (polls && (threadIdx.x & 31) == 0) atomicAdd((int*)polls, 1);
    long long k = 0;
    for (;;) {
        v = w_ld_acquire_cta(p);
        if (__all_sync(kFullMask, v >= need)) {
            cache = __shfl_sync(kFullMask, v, 0);
            return true;
        }
        if (__shfl_sync(kFullMask, *abortFlag, 0)) return false;
        if ((k & 1023) == 1023 && __shfl_sync(kFullMask, *(volatile int*)status, 0) != 0) {
            *abortFlag = 1;
            return false;
        }
        if (++k >= spinMax) {
            if ((threadIdx.x & 31) == 0) atomicExch(status, (int)LUMEN_ERR_TIMEOUT);
            *abortFlag = 1;
            return false;
        }
        // back off: a spinning helper warp would take issue slots from the rows
        __nanosleep(40);
    }
}

// ---- the recurrence (see sgm_step.cuh for the layout and the reference semantics) ----
// Team of T lanes; mpx2: min L' replicated in both halves; p2x2: P2adj
// replicated in both halves.
template <int KW, int T, bool WRAP, bool FULL>
__device__ __forceinline__ void wave_step(const uint32_t (&Lp)[KW], const uint32_t (&Cw)[KW],
                                          uint32_t mpx2, uint32_t p2x2, uint32_t p1x2, uint32_t bsub,
                                          const LaneMasks<KW>& mk, uint32_t (&Ln)[KW]) {
    const uint32_t up = __shfl_up_sync(kFullMask, Lp[KW - 1], 1, T);
    const uint32_t dn = __shfl_down_sync(kFullMask, Lp[0], 1, T);
    uint32_t nb[KW + 1];
    nb[0] = __byte_perm(up, Lp[0], 0x5432);
#pragma unroll
    for (int j = 1; j < KW; ++j) nb[j] = __byte_perm(Lp[j - 1], Lp[j], 0x5432);
    nb[KW] = __byte_perm(Lp[KW - 1], dn, 0x5432);
    if (FULL) {
        nb[0] = (nb[0] & ~mk.nbMask[0]) | (bsub & mk.nbMask[0]);
        nb[KW] = (nb[KW] & ~mk.nbMask[KW]) | (bsub & mk.nbMask[KW]);
    } else {
#pragma unroll
        for (int j = 0; j <= KW; ++j) nb[j] = (nb[j] & ~mk.nbMask[j]) | (bsub & mk.nbMask[j]);
    }
    if (!WRAP) {
        // every valid halfword stays in [0, 65535] (host-proved), so no sum
        // below wraps there.  With P2adj > P1 (the P2 table's floor is P1+1),
        //   min(L', L'[d-1]+P1, L'[d+1]+P1, minL'+P2adj)
        //     = min(min(L'[d-1], L'[d+1], minL'+P2adj-P1) + P1, L')
        // i.e. one three-input minimum and one add-minimum (DPX), then
        // L = m + C - minL' as one IADD3 (m >= minL', no borrow).  Padded halves
        // (d >= D) are overwritten with 0xFFFF below; their garbage borrows only
        // into other padded halves.
        const uint32_t mpp = mpx2 + p2x2 - p1x2;
#pragma unroll
        for (int i = 0; i < KW; ++i) {
            const uint32_t t = __vimin3_u16x2(nb[i], nb[i + 1], mpp);
            const uint32_t m = __viaddmin_u16x2(t, p1x2, Lp[i]);
            uint32_t l = m + Cw[i] - mpx2;
            if (!FULL) l |= mk.padMask[i];
            Ln[i] = l;
        }
    } else {
        const uint32_t mp2 = __vadd2(mpx2, p2x2);
#pragma unroll
        for (int i = 0; i < KW; ++i) {
            const uint32_t c1 = __vadd2(nb[i], p1x2);
            const uint32_t c2 = __vadd2(nb[i + 1], p1x2);
            const uint32_t m = __vminu2(__vminu2(Lp[i], c1), __vminu2(c2, mp2));
            uint32_t l = __vsub2(__vadd2(Cw[i], m), mpx2);
            if (!FULL) l |= mk.padMask[i];
            Ln[i] = l;
        }
    }
}

// min over the warp's disparities, replicated in both halves (gmask: the lanes of the row).
template <int KW>
__device__ __forceinline__ uint32_t wave_min(const uint32_t (&L)[KW], unsigned gmask) {
    uint32_t a[KW];
#pragma unroll
    for (int i = 0; i < KW; ++i) a[i] = L[i];
#pragma unroll
    for (int s = 1; s < KW; s *= 2)
#pragma unroll
        for (int i = 0; i + s < KW; i += 2 * s) a[i] = __vminu2(a[i], a[i + s]);
    const uint32_t m = __vminu2(a[0], __byte_perm(a[0], a[0], 0x1032));
    return __reduce_min_sync(gmask, m);
}

// min over a lane's KW words (per half): three-input minima (DPX) in a
// ternary tree
template <int KW>
__device__ __forceinline__ uint32_t wave_lane_min(const uint32_t (&L)[KW]) {
    uint32_t a[KW];
#pragma unroll
    for (int i = 0; i < KW; ++i) a[i] = L[i];
    int n = KW;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        if (n > 1) {
            int k = 0;
#pragma unroll
            for (int i = 0; i < KW; i += 3) {
                if (i < n) {
                    if (i + 2 < n) a[k] = __vimin3_u16x2(a[i], a[i + 1], a[i + 2]);
                    else if (i + 1 < n) a[k] = __vminu2(a[i], a[i + 1]);
                    else a[k] = a[i];
                    ++k;
                }
            }
            n = k;
        }
    }
    return a[0];
}

// min over a team of T lanes' disparities, replicated in both halves
template <int KW, int T>
__device__ __forceinline__ uint32_t wave_min_t(const uint32_t (&L)[KW]) {
    if constexpr (T == 32) {
        return wave_min<KW>(L, kFullMask);
    } else {
        uint32_t m = wave_lane_min<KW>(L);
        m = __vminu2(m, __byte_perm(m, m, 0x1032));
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) m = __vminu2(m, __shfl_xor_sync(kFullMask, m, o));
        return m;
    }
}

// Warp layout: each row is a team of T lanes (32 / T rows per warp), row
// warps [0, RW), then one import and one export warp.  T = 32 (one row per
// warp) gives the shortest step; narrower teams spread a step's fixed costs
// (prefetch, penalties, addressing, reductions) over several rows and suit
// the throughput-bound batched launches.
template <int KW, bool WRAP, bool FULL, int NP, int R, int T = 32>
__global__ void __launch_bounds__((R / (32 / T) + 2) * 32)
wave_kernel(WaveArgs a) {
    constexpr int LAG = NP == 3 ? 2 : 1;
    constexpr int DP = 2 * KW * T;       // padded disparities
    constexpr int SB = wave_slot_bytes(DP, NP);
    constexpr int RPW = 32 / T;          // rows per warp
    static_assert(R % RPW == 0, "whole warps of rows");
    constexpr int RW = R / RPW;          // row warps
    constexpr int CPV = DP / 16;         // 16-byte cost chunks per pixel
    static_assert(KW % 2 == 0 || CPV <= T, "one cost chunk per team lane");
    extern __shared__ __align__(128) uint8_t sm[];
    const WaveSmem L = wave_smem(a.Wmax, DP, R, NP, a.QI, a.QX);
    const int QI = a.QI, QX = a.QX;
    uint8_t* simg = sm + L.img;
    const uint32_t* p2lut = reinterpret_cast<const uint32_t*>(sm + L.lut);
    // [0] ticket, [1] abort, [2] import polls, [3] export polls, [4] row waits on the helpers
    volatile int* sflag = reinterpret_cast<volatile int*>(sm + L.misc);
    // [0] pixels in the import ring, [1] pixels row 0 no longer needs,
    // [2] pixels in the export ring, [3] pixels the export warp has copied out
    unsigned* sctr = reinterpret_cast<unsigned*>(sm + L.misc) + 8;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tl = lane & (T - 1);  // lane within the row's team
    const int off = tl * 2 * KW;    // first disparity of this lane

    if (threadIdx.x == 0) sflag[1] = 0;
    for (int i = threadIdx.x; i < SB / 4; i += blockDim.x)
        reinterpret_cast<uint32_t*>(sm + L.zero)[i] = 0u;
    __syncthreads();

    LaneMasks<KW> mk;
    int lutP1 = -1, lutP2 = -1, maskD = -1;  // parameters the table and masks were built for

    for (;;) {
        if (threadIdx.x == 0) {
            int t = (int)atomicAdd(a.ticket, 1u);
            if (*(volatile int*)a.status != 0) t = a.nTickets;
            sflag[0] = t;
            sflag[2] = 0; sflag[3] = 0; sflag[4] = 0;
        }
        if (threadIdx.x < 4) sctr[threadIdx.x] = 0u;
        __syncthreads();
        const int t = sflag[0];
        if (t >= a.nTickets) break;
        int sw, b;
        WaveJob J;
        if (a.jobs) {
            const uint32_t e = a.table[t];
            J = a.jobs[e >> 20];
            sw = (e >> 19) & 1;
            b = (int)(e & 0x7FFFFu);
        } else {
            J = a.job;
            sw = t & 1;
            b = t >> 1;
        }
        const bool active = b < J.nBands;
        const int tb = t;  // band ticket (trace record, stall test)
        const int W = J.W, H = J.H;
        if (J.P1 != lutP1 || J.P2 != lutP2) {
            // adaptive P2 (src/sgbm_kernels.cu:301-310) as a table of |dI|, replicated in both halves
            for (int g = threadIdx.x; g < 256; g += blockDim.x)
                reinterpret_cast<uint32_t*>(sm + L.lut)[g] =
                    ((uint32_t)max(J.P1 + 1, J.P2 * 8 / max(8, g)) & 0xFFFFu) * 0x10001u;
            lutP1 = J.P1;
            lutP2 = J.P2;
        }
        if (J.D != maskD) {
            make_lane_masks<KW>(tl, J.D, mk);
            maskD = J.D;
        }
        const int v0 = b * R;
        const int lastActive = min(R - 1, H - 1 - v0);
        const bool hasPrev = b > 0, hasNext = b + 1 < J.nBands;
        const bool globalImport = hasPrev, globalExport = hasNext;
        // ---- stage sweep-oriented image rows v0-1 .. v0+R-1 ----
        for (int i = threadIdx.x; i < (active ? (R + 1) * W : 0); i += blockDim.x) {
            const int rr = i / W, u = i - rr * W;
            const int vv = v0 - 1 + rr;
            uint8_t val = 0;
            if (vv >= 0 && vv < H) {
                const int x = sw ? W - 1 - u : u, y = sw ? H - 1 - vv : vv;
                val = J.img[(size_t)y * W + x];
            }
            simg[rr * L.Wp + u] = val;
        }
        const unsigned stallPix = (a.stallTest && tb == 2) ? (unsigned)W + 1u : 0u;
        bool ok = true;
        __syncthreads();
        // [24..27]: globaltimer of the middle pixel in the first and the last row
        unsigned long long* tMid = reinterpret_cast<unsigned long long*>(sm + L.misc) + 12;

        if (!active) {
            // no band for this rank in this ticket
        } else if (warp < RW) {
            // ===================== row warps, lockstep =====================
            const int r = warp * RPW + lane / T;           // this team's row
            const bool rowOn = r <= lastActive;
            const int v = v0 + min(r, lastActive);
            const int y = sw ? H - 1 - v : v;
            const bool startV = (v0 + r == 0);
            const bool exporter = rowOn && r == lastActive && hasNext;
            const bool writes = rowOn && (r < lastActive || exporter);
            const bool importer0 = (r == 0) && hasPrev;
            uint8_t* const ringIn = r == 0 ? (sm + L.imp) : (sm + L.rings + (r - 1) * kWQ * SB);
            const int pQm = (r == 0 ? QI : kWQ) - 1;
            uint8_t* const ringOut = exporter ? (sm + L.exp) : (sm + L.rings + min(r, R - 2) * kWQ * SB);
            const int oQm = (exporter ? QX : kWQ) - 1;
            const uint8_t* const zeroSlot = sm + L.zero;
            uint8_t* const costRing = sm + L.cost + r * kWPF * DP;
            const uint8_t* irow = simg + (r + 1) * L.Wp;
            const uint8_t* iprev = simg + r * L.Wp;
            uint16_t* pout = (sw ? J.part[1] : J.part[0]) + ((size_t)y * W + (sw ? W - 1 : 0)) * DP + off;
            const ptrdiff_t pstep = sw ? -(ptrdiff_t)DP : (ptrdiff_t)DP;
            // Cost prefetch: when a lane's 2*KW cost bytes are a multiple of 4 it
            // copies exactly its own bytes (no cross-lane dependency); otherwise
            // the first DP/16 lanes copy 16-byte chunks and the warp syncs.
            constexpr bool OWN = (KW % 2) == 0;
            const uint8_t* cgrow = J.cost + (size_t)y * W * DP;
            auto prefetch = [&](int step) {
                const int p = step - LAG * r + kWPF - 1;
                if (rowOn && p >= 0 && p < W) {
                    const int x = sw ? W - 1 - p : p;
                    const uint8_t* src = cgrow + (size_t)x * DP;
                    const uint32_t dst = w_smem_addr(costRing + (p % kWPF) * DP);
                    if constexpr (OWN && (2 * KW) % 16 == 0) {
#pragma unroll
                        for (int q = 0; q < (2 * KW) / 16; ++q) w_cp_async16(dst + off + 16 * q, src + off + 16 * q);
                    } else if (OWN) {
#pragma unroll
                        for (int q = 0; q < KW / 2; ++q)
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + off + 4 * q),
                                         "l"(src + off + 4 * q)
                                         : "memory");
                    } else if (tl < CPV) {
                        w_cp_async16(dst + 16 * tl, src + 16 * tl);
                    }
                }
                w_cp_commit();
            };
            for (int s = -(kWPF - 1); s < 0; ++s) prefetch(s);

            const int nSteps = W + LAG * lastActive;
            uint32_t LH[KW];
#pragma unroll
            for (int w = 0; w < KW; ++w) LH[w] = 0;
            uint32_t minH = 0;
            unsigned impSeen = 0, expSeen = 0;
            // the helper waits take whole warps: the one holding row 0 (imports)
            // and the one holding the exporting row (export ring space)
            const bool warpImports = hasPrev && warp == 0;
            const bool warpExports = hasNext && warp == lastActive / RPW;
            for (int step = 0; step < nSteps; ++step) {
                const int u = step - LAG * r;
                const bool on = rowOn && u >= 0 && u < W;
                const int uc = min(max(u, 0), W - 1);
                // ---- helper hand-offs (row 0 / the exporting row) ----
                const int u0 = step, uE = step - LAG * lastActive;  // row 0's and the exporting row's pixel
                if (warpImports && ok && u0 < W)
                    ok = w_wait_cta(&sctr[0], (unsigned)min(W, u0 + 2), impSeen, sflag + 1, a.status,
                                    a.spinMax, a.trace ? sflag + 4 : nullptr);
                if (warpExports && ok && uE >= QX && uE < W)
                    ok = w_wait_cta(&sctr[3], (unsigned)(uE - QX + 1), expSeen, sflag + 1, a.status,
                                    a.spinMax, a.trace ? sflag + 4 : nullptr);
                // ---- cost of this step's pixel ----
                prefetch(step);
                w_cp_wait<kWPF - 1>();
                if (!OWN) __syncwarp();
                uint32_t Cw[KW];
                load_cost_words<KW>(costRing + (uc % kWPF) * DP + off, Cw);
                if (WRAP || J.costScale != 1) {
#pragma unroll
                    for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(Cw[w], J.costScale);
                }
                // ---- adaptive P2 of this pixel: H path, V, D1 (u-1, v-1), D2 (u+1, v-1) ----
                const int cur = irow[uc];
                const uint32_t p2h = p2lut[abs(cur - irow[max(uc - 1, 0)])];
                const uint32_t p2v[3] = {p2lut[abs(cur - iprev[uc])], p2lut[abs(cur - iprev[max(uc - 1, 0)])],
                                         p2lut[abs(cur - iprev[min(uc + 1, W - 1)])]};
                // ---- horizontal path ----
                uint32_t LnH[KW];
                wave_step<KW, T, WRAP, FULL>(LH, Cw, minH, p2h, J.p1x2, J.bsub, mk, LnH);
                // ---- vertical / diagonal paths from the previous row ----
                uint32_t Ln[NP][KW], mn[NP];
#pragma unroll
                for (int pth = 0; pth < NP; ++pth) {
                    const int pu = pth == 0 ? uc : (pth == 1 ? uc - 1 : uc + 1);
                    const bool zero = startV || pu < 0 || pu >= W;
                    const uint8_t* slot = zero ? zeroSlot : ringIn + (pu & pQm) * SB;
                    uint32_t Lp[KW];
                    load_words<KW>(reinterpret_cast<const uint16_t*>(slot + pth * 2 * DP) + off, Lp);
                    const uint32_t mp = reinterpret_cast<const uint32_t*>(slot + NP * 2 * DP)[pth];
                    wave_step<KW, T, WRAP, FULL>(Lp, Cw, mp, p2v[pth], J.p1x2, J.bsub, mk, Ln[pth]);
                }
                // a row that has not reached its first pixel ran on dummy data: its
                // horizontal-path state must stay at its start value (0)
                const uint32_t minHn = wave_min_t<KW, T>(LnH);
                minH = on ? minHn : minH;
#pragma unroll
                for (int pth = 0; pth < NP; ++pth) mn[pth] = wave_min_t<KW, T>(Ln[pth]);
                uint32_t S[KW];
#pragma unroll
                for (int w = 0; w < KW; ++w) {
                    LH[w] = on ? LnH[w] : LH[w];
                    uint32_t sum = LnH[w];
#pragma unroll
                    for (int pth = 0; pth < NP; ++pth) sum = WRAP ? __vadd2(sum, Ln[pth][w]) : sum + Ln[pth][w];
                    S[w] = sum;
                }
                if (a.trace && tl == 0 && on && u == (W >> 1)) {
                    if (r == 0) tMid[0] = wave_now();
                    if (r == lastActive) tMid[1] = wave_now();
                }
                if (on && ok) {
                    store_words<KW>(pout, S);
                    pout += pstep;
                    // ---- hand the vertical-type vectors to the next row / the export warp ----
                    if (writes) {
                        uint8_t* slot = ringOut + (u & oQm) * SB;
#pragma unroll
                        for (int pth = 0; pth < NP; ++pth)
                            store_words<KW>(reinterpret_cast<uint16_t*>(slot + pth * 2 * DP) + off, Ln[pth]);
                        if (tl == 0) {
                            if (NP == 3)
                                *reinterpret_cast<uint4*>(slot + NP * 2 * DP) = make_uint4(mn[0], mn[NP > 1 ? 1 : 0], mn[NP > 2 ? 2 : 0], 0u);
                            else
                                *reinterpret_cast<uint32_t*>(slot + NP * 2 * DP) = mn[0];
                        }
                    }
                }
                // publish the exporting row's slot and row 0's progress (every
                // lane of the warp has stored its part of the slot)
                if (warpImports || warpExports) {
                    __syncwarp();
                    if (tl == 0 && on && ok) {
                        if (exporter) w_st_release_cta(&sctr[2], (unsigned)(u + 1));
                        if (importer0) w_st_release_cta(&sctr[1], (unsigned)u);
                    }
                }
                if (RW > 1) w_rows_barrier(RW * 32);
                else __syncwarp();
            }
            w_cp_wait<0>();
        } else if (warp == RW) {
            // ===================== import warp: previous band's last row =====================
            if (globalImport) {
                const uint8_t* xin = J.xring + ((size_t)(sw * J.nBands + b - 1) * kWK) * SB;
                const unsigned* iprod = J.prod + sw * J.nBands + (b - 1);
                unsigned* icons = J.cons + sw * J.nBands + (b - 1);
                unsigned prodSeen = 0, r0Seen = 0;
                const uint32_t impA = w_smem_addr(sm + L.imp);
                for (int p = 0; p < W && ok; ++p) {
                    if (p >= QI)
                        ok = w_wait_cta(&sctr[1], (unsigned)(p - QI + 1), r0Seen, sflag + 1, a.status, a.spinMax);
                    if (ok)
                        ok = w_wait_gpu(iprod, stallPix ? stallPix : (unsigned)(p + 1), prodSeen, sflag + 1,
                                        a.status, a.spinMax, lane, a.trace ? sflag + 2 : nullptr);
                    if (!ok) break;
                    const uint8_t* src = xin + (size_t)(p & (kWK - 1)) * SB;
                    const uint32_t dst = impA + (p & (QI - 1)) * SB;
                    for (int i = lane; i < SB / 16; i += 32) w_cp_async16(dst + 16 * i, src + 16 * i);
                    w_cp_commit();
                    if (p >= 2) {
                        w_cp_wait<2>();
                        __syncwarp();
                        const int done = p - 1;
                        if (lane == 0) {
                            w_st_release_cta(&sctr[0], (unsigned)done);
                            if ((done % kWE) == 0) w_st_release_gpu(icons, (unsigned)done);
                        }
                    }
                }
                w_cp_wait<0>();
                __syncwarp();
                if (ok && lane == 0) {
                    w_st_release_cta(&sctr[0], (unsigned)W);
                    w_st_release_gpu(icons, (unsigned)W);
                }
            }
        } else {
            // ===================== export warp: this band's last row =====================
            if (globalExport) {
                uint8_t* xout = J.xring + ((size_t)(sw * J.nBands + b) * kWK) * SB;
                unsigned* oprod = J.prod + sw * J.nBands + b;
                const unsigned* ocons = J.cons + sw * J.nBands + b;
                unsigned availSeen = 0, consSeen = 0;
                for (int u = 0; u < W && ok; ++u) {
                    ok = w_wait_cta(&sctr[2], (unsigned)(u + 1), availSeen, sflag + 1, a.status, a.spinMax);
                    if (ok && u >= kWK)
                        ok = w_wait_gpu(ocons, (unsigned)(u - kWK + 1), consSeen, sflag + 1, a.status,
                                        a.spinMax, lane, a.trace ? sflag + 3 : nullptr);
                    if (!ok) break;
                    const uint4* src = reinterpret_cast<const uint4*>(sm + L.exp + (u & (QX - 1)) * SB);
                    uint4* dst = reinterpret_cast<uint4*>(xout + (size_t)(u & (kWK - 1)) * SB);
                    for (int i = lane; i < SB / 16; i += 32) __stcg(dst + i, src[i]);
                    __syncwarp();
                    if (lane == 0) {
                        w_st_release_cta(&sctr[3], (unsigned)(u + 1));
                        if (((u + 1) % kWE) == 0 || u == W - 1) w_st_release_gpu(oprod, (unsigned)(u + 1));
                    }
                }
            }
        }
        const bool stop = __syncthreads_or(!ok || sflag[1] != 0);
        if (a.trace && active && threadIdx.x == 0) {
            unsigned smid;
            asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
            unsigned long long* rec = a.trace + 4 * (size_t)tb;
            rec[0] = tMid[0];
            rec[1] = tMid[1];
            rec[2] = wave_now();
            auto sat = [](int x) { return (unsigned long long)min(x, 0xFFFF); };
            rec[3] = ((unsigned long long)smid << 48) | (sat(sflag[2]) << 32) | (sat(sflag[3]) << 16) |
                     sat(sflag[4]);
        }
        if (stop) break;
    }
}

}  // namespace lumen
