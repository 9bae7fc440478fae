// pair_kernel.cuh -- SGM aggregation as four lag-free sweeps (schedule 6).
//
// The eight path kernels of the reference (src/sgbm_kernels.cu:315-742) regroup
// into four sweeps of two paths each: one horizontal path of the sweep and the
// one diagonal that runs the same way.  In sweep coordinates (u along a sweep
// row, v across rows) both paths of a pixel (u, v) come from pixel u-1:
//   sweep 0  rows top-down,     pixels left-to-right   LR   (u-1, v)  TLBR (u-1, v-1)
//   sweep 1  rows bottom-up,    pixels right-to-left   RL              BRTL
//   sweep 2  columns right-to-left, pixels top-down    TB              TRBL
//   sweep 3  columns left-to-right, pixels bottom-up   BT              BLTR
// with (x, y) = (u, v), (W-1-u, H-1-v), (W-1-v, u), (v, H-1-u).  Sweeps 2 and
// 3 run over the columns of the image: their "rows" are image columns.
//
// Because row v needs only pixel u-1 of row v-1, all rows of a band handle
// the same pixel at the same step (no lag between rows): a band of R rows
// spans its row length in steps, and the next band trails it by one
// hand-off, so a sweep spans about len + bands * hand-off steps instead of
// the W + 2H of a sweep that also carries TRBL.
//
// Work decomposition:
//  * a CTA owns a band of R consecutive sweep rows, each row a team of T
//    lanes (a lane holds 2*KW disparities as KW packed uint16x2 words); the
//    row warps advance in lockstep, one barrier per step, which also takes
//    the OR of every row's stop request so all rows leave at the same step;
//  * row r reads row r-1's diagonal vector of pixel u-1 from a two-slot
//    shared-memory ring written one step earlier;
//  * the band's last row writes its diagonal vector of every pixel into a
//    per-boundary row buffer in global memory as 64-bit (payload, epoch)
//    words, plain stores with no fence: a word is valid once its high half
//    holds this launch's epoch.  The producing rows never wait on global
//    memory;
//  * an import warp outside the row barrier probes one word of the band
//    above's next pixel (backing off while nothing arrives), then loads up to
//    kPG pixels, copies every leading pixel whose words all carry the epoch
//    into a kPQ-slot shared-memory ring and publishes the count (release at
//    CTA scope); row 0 takes pixel u-1 from that ring at step u.  After
//    each step's barrier the rows publish how many pixels row 0 has consumed,
//    which frees ring slots.  The row buffers hold whole rows, so a band
//    waits only on the band above it, never on the one below: bands depend
//    only on earlier tickets and any number of resident CTAs makes progress;
//  * matching costs are prefetched kPPF-1 pixels ahead with cp.async;
//    adaptive P2 is looked up from staged image rows;
//  * bands are handed out by a ticket counter, the four sweeps interleaved,
//    each sweep's bands in order.  A batched launch (PairArgs::jobs) takes
//    its tickets from a table over the bands of many pairs of one kernel
//    class; a CTA copies each band's pair descriptor into shared memory and
//    rebuilds the P2 table and lane masks when the pair changes.
// Every wait is bounded: on timeout the CTA records LUMEN_ERR_TIMEOUT in
// *status and stops; CTAs that see a non-zero status stop taking bands.
#pragma once

#include "pair_layout.h"
#include "wave_kernel.cuh"

namespace lumen {

struct PairJob {
    const uint8_t* cost;           // [H][W][Dp]
    const uint8_t* img;            // [H][W] left gray image (adaptive P2)
    uint16_t* part[4];             // per-sweep partial sums, [H][W][Dp]
    unsigned long long* xbuf;      // band-boundary rows: pair_ll_words(Dp) words a pixel (pair_xbase)
    int W, H, D;
    int nb[2];                     // bands of the row sweeps (0, 1) and of the column sweeps (2, 3)
    int P1, P2, costScale;
    uint32_t p1x2, bsub;
};

// Descriptor of one pair (host side, pair.cu): its volumes, row buffers
// (8 paths), sizes, bands for R rows per band, and parameters.
PairJob pair_job(const PairView& pv, uint16_t* const part[4], const SgmConsts& k, int R,
                 unsigned long long* xbuf);

// A launch: one pair (`job`, tickets through pair_ticket) or a batch of pairs
// of one kernel class (`jobs`, tickets through `table`, each entry
// pair << 20 | sweep << 18 | band, every band listed after the band before it
// in its own sweep).
struct PairArgs {
    PairJob job;                   // the pair when jobs == nullptr
    const PairJob* jobs;           // batch: [pairs]
    const uint32_t* table;         // batch: [nTickets]
    int nTickets;                  // one pair: 2 * nb[0] + 2 * nb[1]
    int Lmax;                      // max(W, H) over the launch's pairs: staged image row length
    unsigned* ticket;
    int* status;
    long long spinMax;
    unsigned epoch;                // high half of every row-buffer word this launch writes
    int sweeps;                    // one pair: 0 all four sweeps, 1 the row sweeps (0, 1), 2 the column sweeps (2, 3)
    int stallTest;                 // 1: band 1 of sweep 0 waits for an epoch never written
    unsigned long long* trace;     // optional band timeline, [nTickets][4] (pair_trace_record)
};

// Band timeline record (lumen_sgbm_debug_trace) of schedule 6, per ticket:
// [0] globaltimer ns when the band's rows start their first pixel, [1] when
// they have finished pixel len/2, [2] when they have finished the row, [3] the
// SM id << 32 | the sweep << 16 | 1.  Consecutive bands' [1] give the
// hand-off lag; ([2] - [0]) / len the time of one step.
__device__ __forceinline__ unsigned long long pair_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// 64-bit (payload, epoch) words of the row buffers: volatile accesses reach
// the GPU-wide L2 and each 64-bit element is single-copy atomic, so a reader
// sees a word either from an earlier launch or complete from this one.
__device__ __forceinline__ void ll_store2(unsigned long long* p, unsigned long long a, unsigned long long b) {
    asm volatile("st.volatile.global.v2.u64 [%0], {%1, %2};\n" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ void ll_load2(const unsigned long long* p, unsigned long long& a,
                                         unsigned long long& b) {
    asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];\n" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}

// Named barrier 1 over the row warps' threads with an OR reduction: every
// row thread gets the OR of all of their `v`.
__device__ __forceinline__ bool rows_barrier_or(int nThreads, bool v) {
    uint32_t r;
    asm volatile(
        "{\n"
        " .reg .pred p, q;\n"
        " setp.ne.u32 p, %1, 0;\n"
        " bar.red.or.pred q, 1, %2, p;\n"
        " selp.u32 %0, 1, 0, q;\n"
        "}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(nThreads)
        : "memory");
    return r != 0;
}

// DIAG = false: the four paths LR, RL, TB, BT alone (4-path mode).  Then no
// row depends on another: bands have no import warp, no hand-off and no
// per-step barrier, every row warp runs free.
template <int KW, bool WRAP, bool FULL, int R, int T, bool DIAG>
__device__ __forceinline__ void pair_body(const PairArgs& a) {
    constexpr int DP = 2 * KW * T;       // padded disparities
    constexpr int SB = pair_slot_bytes(DP);
    constexpr int NL = pair_ll_words(DP);
    constexpr int PAIRS = NL / 2;        // 16-byte pairs of row-buffer words a pixel
    constexpr int RPW = 32 / T;          // rows per warp
    static_assert(R % RPW == 0, "whole warps of rows");
    constexpr int RW = R / RPW;          // row warps; warp RW imports
    static_assert(KW % 2 == 0, "a lane's cost bytes are whole 4-byte words; its words pair up");
    static_assert((kPQ & (kPQ - 1)) == 0 && kPG <= kPQ && kPG <= 32, "import ring");
    extern __shared__ __align__(128) uint8_t sm[];
    const PairSmem L = pair_smem(a.Lmax, DP, R);
    uint8_t* simg = sm + L.img;
    const uint32_t* p2lut = reinterpret_cast<const uint32_t*>(sm + L.lut);
    // [0] ticket, [1] abort
    volatile int* sflag = reinterpret_cast<volatile int*>(sm + L.misc);
    // [0] pixels of the band above in the import ring, [1] pixels row 0 has consumed
    unsigned* sctr = reinterpret_cast<unsigned*>(sm + L.misc) + 8;
    const uint8_t* const zeroSlot = sm + L.zero;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tl = lane & (T - 1);      // lane within the row's team
    const int off = tl * 2 * KW;        // first disparity of this lane
    const int r = warp * RPW + lane / T;

    for (int i = threadIdx.x; i < SB / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sm + L.zero)[i] = 0u;
    LaneMasks<KW> mk;
    int curJob = -1;   // the pair whose P2 table and lane masks are set up
    // the band's pair, copied from the launch's parameters or job table
    PairJob* const sJob = reinterpret_cast<PairJob*>(sm + L.job);
    static_assert(sizeof(PairJob) <= kPairJobBytes, "pair descriptor slot");

    for (;;) {
        if (threadIdx.x == 0) {
            int t = (int)atomicAdd(a.ticket, 1u);
            if (*(volatile int*)a.status != 0) t = a.nTickets;
            sflag[0] = t;
            sflag[1] = 0;
            if (t < a.nTickets) {
                int s, b, jb = 0;
                if (a.jobs) {
                    const uint32_t e = a.table[t];
                    jb = (int)(e >> 20);
                    s = (int)(e >> 18) & 3;
                    b = (int)(e & 0x3FFFFu);
                    *sJob = a.jobs[jb];
                } else {
                    if (a.sweeps == 0) {
                        pair_ticket(t, a.job.nb[0], a.job.nb[1], s, b);
                    } else {   // two sweeps of one kind, bands in order
                        s = (a.sweeps == 1 ? 0 : 2) + (t & 1);
                        b = t >> 1;
                    }
                    if (curJob < 0) *sJob = a.job;
                }
                sflag[2] = s;
                sflag[3] = b;
                sflag[4] = jb;
            }
        }
        if (threadIdx.x < 2) sctr[threadIdx.x] = 0u;
        __syncthreads();
        const int t = sflag[0];
        if (t >= a.nTickets) break;
        const int s = sflag[2], b = sflag[3], jb = sflag[4];
        const PairJob& J = *sJob;
        const int W = J.W, H = J.H;
        if (jb != curJob) {
            // adaptive P2 (src/sgbm_kernels.cu:301-310) as a table of |dI|, replicated
            // in both halves (read after the staging barrier below)
            for (int g = threadIdx.x; g < 256; g += blockDim.x)
                reinterpret_cast<uint32_t*>(sm + L.lut)[g] =
                    ((uint32_t)max(J.P1 + 1, J.P2 * 8 / max(8, g)) & 0xFFFFu) * 0x10001u;
            make_lane_masks<KW>(tl, J.D, mk);
            curJob = jb;
        }
        const bool tr = s >= 2;
        const int Ws = tr ? H : W, Hs = tr ? W : H;
        const int nbS = tr ? J.nb[1] : J.nb[0];
        const int v0 = b * R;
        const int lastActive = min(R - 1, Hs - 1 - v0);
        const bool hasPrev = DIAG && b > 0, hasNext = DIAG && b + 1 < nbS;
        // ---- stage sweep rows v0-1 .. v0+R-1 of the image (column sweeps: row index fastest) ----
        for (int i = threadIdx.x; i < (R + 1) * Ws; i += blockDim.x) {
            int rr, u;
            if (tr) { rr = i % (R + 1); u = i / (R + 1); }
            else { rr = i / Ws; u = i - rr * Ws; }
            const int vv = v0 - 1 + rr;
            uint8_t val = 0;
            if (vv >= 0 && vv < Hs) {
                int x, y;
                pair_xy(s, u, vv, W, H, x, y);
                val = J.img[(size_t)y * W + x];
            }
            simg[rr * L.Lp + u] = val;
        }
        __syncthreads();
        bool ok = true;

        if (warp < RW) {
            // ===================== row warps, lockstep =====================
            const bool rowOn = r <= lastActive;
            const int v = v0 + min(r, lastActive);
            int x0, y0;
            pair_xy(s, 0, v, W, H, x0, y0);
            const ptrdiff_t du = s == 0 ? 1 : s == 1 ? -1 : s == 2 ? (ptrdiff_t)W : -(ptrdiff_t)W;
            const ptrdiff_t pix0 = (ptrdiff_t)y0 * W + x0;
            uint16_t* const part = s == 0 ? J.part[0] : s == 1 ? J.part[1] : s == 2 ? J.part[2] : J.part[3];
            uint16_t* pout = part + pix0 * DP + off;
            const ptrdiff_t pstep = du * DP;
            uint8_t* const costRing = sm + L.cost + r * kPPF * DP;
            const uint8_t* irow = simg + (r + 1) * L.Lp;
            const uint8_t* iprev = simg + r * L.Lp;
            uint8_t* const mySlots = sm + L.slots + r * 2 * SB;
            const uint8_t* const upSlots = sm + L.slots + (r > 0 ? r - 1 : 0) * 2 * SB;
            const uint8_t* const impRing = sm + L.imp;
            const bool exporter = rowOn && r == lastActive && hasNext;
            unsigned long long* xo =
                exporter ? J.xbuf + pair_xbase(s, b, W, H, J.nb[0], J.nb[1]) * NL + tl * KW : nullptr;
            const unsigned long long ep = (unsigned long long)a.epoch << 32;
            // the pair's fields the steps use, in registers
            const uint8_t* const costBase = J.cost;
            const int costScale = J.costScale;
            const uint32_t p1x2 = J.p1x2, bsub = J.bsub;

            if constexpr (!DIAG) {
                // one path a sweep, rows independent: costs arrive in batches of
                // four pixels (one cp.async group a batch; batch q holds pixels
                // 4q .. 4q+3 in ring slots p % kPPF, the ring holds two batches),
                // and pixel u+1's cost words and P2 value are loaded during step
                // u, before its reduction, so their latency overlaps the shuffles
                static_assert(kPPF == 8, "two batches of four pixels");
                ptrdiff_t qofs = pix0 * DP + off;   // bytes from J.cost of the next batch's first pixel
                const ptrdiff_t qstep = du * DP;
                auto prefetch_batch = [&](int q) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int p = 4 * q + k;
                        if (rowOn && p < Ws) {
                            const uint8_t* src = costBase + (qofs + k * qstep);
                            const uint32_t dst = w_smem_addr(costRing + (p % kPPF) * DP + off);
                            if constexpr ((2 * KW) % 16 == 0) {
#pragma unroll
                                for (int c = 0; c < (2 * KW) / 16; ++c) w_cp_async16(dst + 16 * c, src + 16 * c);
                            } else {
#pragma unroll
                                for (int c = 0; c < KW / 2; ++c)
                                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 4 * c),
                                                 "l"(src + 4 * c)
                                                 : "memory");
                            }
                        }
                    }
                    qofs += 4 * qstep;
                    w_cp_commit();
                };
                uint32_t Cw[KW];
                uint32_t p2h;
                auto load_operands = [&](int u) {
                    load_cost_words<KW>(costRing + (u % kPPF) * DP + off, Cw);
                    if (WRAP || costScale != 1) {
#pragma unroll
                        for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(Cw[w], costScale);
                    }
                    p2h = p2lut[abs(irow[u] - irow[max(u - 1, 0)])];
                };
                prefetch_batch(0);
                prefetch_batch(1);
                w_cp_wait<1>();
                load_operands(0);
                uint32_t LH[KW];
#pragma unroll
                for (int w = 0; w < KW; ++w) LH[w] = 0;
                uint32_t minH = 0;
                for (int u = 0; u < Ws; ++u) {
                    uint32_t LnH[KW];
                    wave_step<KW, T, WRAP, FULL>(LH, Cw, minH, p2h, p1x2, bsub, mk, LnH);
                    if (u + 1 < Ws) {
                        if ((u & 3) == 3) {
                            prefetch_batch((u >> 2) + 2);   // into the slots of pixels u-3 .. u, all read
                            w_cp_wait<1>();                 // batch (u >> 2) + 1, pixels u+1 .. u+4, has landed
                        }
                        load_operands(u + 1);
                    }
                    minH = wave_min_t<KW, T>(LnH);
#pragma unroll
                    for (int w = 0; w < KW; ++w) LH[w] = LnH[w];
                    if (rowOn) {
                        store_words<KW>(pout, LnH);
                        pout += pstep;
                    }
                }
                w_cp_wait<0>();
            } else {
            // cost of pixel p = step + kPPF - 1 of this row: `cofs` (bytes from
            // J.cost) follows p, incremented instead of recomputed; the calls
            // come with step = -(kPPF - 1), -(kPPF - 2), ..., i.e. p = 0, 1, ...
            ptrdiff_t cofs = pix0 * DP + off;
            const ptrdiff_t cstep = du * DP;
            auto prefetch = [&](int step) {
                const int p = step + kPPF - 1;
                const ptrdiff_t o = cofs;
                cofs += cstep;
                if (rowOn && p >= 0 && p < Ws) {
                    const uint8_t* src = costBase + o;
                    const uint32_t dst = w_smem_addr(costRing + (p % kPPF) * DP + off);
                    if constexpr ((2 * KW) % 16 == 0) {
#pragma unroll
                        for (int q = 0; q < (2 * KW) / 16; ++q) w_cp_async16(dst + 16 * q, src + 16 * q);
                    } else {
#pragma unroll
                        for (int q = 0; q < KW / 2; ++q)
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 4 * q),
                                         "l"(src + 4 * q)
                                         : "memory");
                    }
                }
                w_cp_commit();
            };
            for (int st = -(kPPF - 1); st < 0; ++st) prefetch(st);

            uint32_t LH[KW];
#pragma unroll
            for (int w = 0; w < KW; ++w) LH[w] = 0;
            uint32_t minH = 0;
            unsigned impSeen = 0;
            unsigned long long* const trec = (a.trace && threadIdx.x == 0) ? a.trace + 4 * (size_t)t : nullptr;
            if (trec) trec[0] = pair_now();
            for (int u = 0; u < Ws; ++u) {
                // ---- the band above's pixel u-1 must be in the import ring (warp 0 holds row 0) ----
                if (warp == 0 && hasPrev && u >= 1 && ok)
                    ok = w_wait_cta(&sctr[0], (unsigned)u, impSeen, sflag + 1, a.status, a.spinMax);
                // ---- cost of this step's pixel ----
                prefetch(u);
                w_cp_wait<kPPF - 1>();
                uint32_t Cw[KW];
                load_cost_words<KW>(costRing + (u % kPPF) * DP + off, Cw);
                if (WRAP || costScale != 1) {
#pragma unroll
                    for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(Cw[w], costScale);
                }
                // ---- adaptive P2: horizontal predecessor (u-1, v), diagonal (u-1, v-1) ----
                const int um = max(u - 1, 0);
                const int cur = irow[u];
                const uint32_t p2h = p2lut[abs(cur - irow[um])];
                // ---- horizontal path (its state starts at 0: L = C at u = 0) ----
                uint32_t LnH[KW];
                wave_step<KW, T, WRAP, FULL>(LH, Cw, minH, p2h, p1x2, bsub, mk, LnH);
                const uint32_t p2d = p2lut[abs(cur - iprev[um])];
                // ---- diagonal path from the row above, pixel u-1 ----
                const uint8_t* slot = (u == 0 || v == 0) ? zeroSlot
                                      : r == 0           ? impRing + ((u - 1) & (kPQ - 1)) * SB
                                                         : upSlots + ((u - 1) & 1) * SB;
                uint32_t Lp[KW];
                load_words<KW>(reinterpret_cast<const uint16_t*>(slot) + off, Lp);
                const uint32_t mp = *reinterpret_cast<const uint32_t*>(slot + 2 * DP);
                uint32_t LnD[KW];
                wave_step<KW, T, WRAP, FULL>(Lp, Cw, mp, p2d, p1x2, bsub, mk, LnD);
                minH = wave_min_t<KW, T>(LnH);
                const uint32_t minD = wave_min_t<KW, T>(LnD);
                uint32_t S[KW];
#pragma unroll
                for (int w = 0; w < KW; ++w) {
                    LH[w] = LnH[w];
                    S[w] = WRAP ? __vadd2(LnH[w], LnD[w]) : LnH[w] + LnD[w];
                }
                // ---- hand the diagonal vector to the row below / the band below ----
                {
                    uint8_t* my = mySlots + (u & 1) * SB;
                    store_words<KW>(reinterpret_cast<uint16_t*>(my) + off, LnD);
                    if (tl == 0) *reinterpret_cast<uint32_t*>(my + 2 * DP) = minD;
                }
                if (rowOn) {
                    store_words<KW>(pout, S);
                    pout += pstep;
                    if (exporter) {
#pragma unroll
                        for (int w = 0; w < KW; w += 2) ll_store2(xo + w, ep | LnD[w], ep | LnD[w + 1]);
                        if (tl == 0) ll_store2(xo + DP / 2, ep | minD, ep);   // the minimum and the pad word
                        xo += NL;
                    }
                }
                // every row has finished step u (row 0 is done with pixel u-1 of the
                // import ring); all rows stop together when any of them must
                if (rows_barrier_or(RW * 32, !ok || sflag[1] != 0)) {
                    ok = false;
                    break;
                }
                if (threadIdx.x == 0 && hasPrev) w_st_release_cta(&sctr[1], (unsigned)u);
                if (trec && u == Ws / 2) trec[1] = pair_now();
            }
            if (trec) {
                unsigned smid;
                asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
                trec[2] = pair_now();
                trec[3] = (unsigned long long)smid << 32 | (unsigned)s << 16 | 1u;
            }
            w_cp_wait<0>();
            }
        } else if (hasPrev) {
            // ===================== import warp: the band above's last row =====================
            const unsigned long long* xin = J.xbuf + pair_xbase(s, b - 1, W, H, J.nb[0], J.nb[1]) * NL;
            const unsigned want = (a.stallTest && s == 0 && b == 1) ? a.epoch + 1u : a.epoch;
            const int nImp = Ws - 1;     // row 0 uses pixels 0 .. Ws-2
            constexpr int PER = (kPG * PAIRS + 31) / 32;
            unsigned freeSeen = 0;
            long long spins = 0;
            unsigned nap = 32;   // back-off between probes (ns), doubled while nothing arrives
            int p0 = 0;
            while (p0 < nImp && ok) {
                const int g = min(kPG, nImp - p0);
                // ring space: pixel p replaces pixel p - kPQ, which row 0 must have consumed
                if (p0 + g > kPQ)
                    ok = w_wait_cta(&sctr[1], (unsigned)(p0 + g - kPQ), freeSeen, sflag + 1, a.status, a.spinMax);
                if (!ok) break;
                // probe: one lane reads pixel p0's minimum word; the full load and
                // check of up to kPG pixels follows only once it carries the epoch,
                // so a waiting import warp takes few issue slots from the rows
                unsigned long long pa = 0, pb = 0;
                if (lane == 0) ll_load2(xin + (size_t)p0 * NL + DP / 2, pa, pb);
                if (!__shfl_sync(kFullMask, (unsigned)(pa >> 32) == want ? 1u : 0u, 0)) {
                    if (sflag[1]) {
                        ok = false;
                        break;
                    }
                    if ((spins & 63) == 63 && *(volatile int*)a.status != 0) {
                        sflag[1] = 1;
                        ok = false;
                        break;
                    }
                    if (++spins >= a.spinMax) {
                        if (lane == 0) atomicExch(a.status, (int)LUMEN_ERR_TIMEOUT);
                        sflag[1] = 1;
                        ok = false;
                        break;
                    }
                    __nanosleep(nap);
                    nap = min(nap * 2u, 256u);
                    continue;
                }
                unsigned long long va[PER], vb[PER];
                unsigned bad = 0;   // pixels (bit g') with a word not yet written by this launch
#pragma unroll
                for (int j = 0; j < PER; ++j) {
                    const int f = lane + 32 * j;
                    const int px = f / PAIRS, q = f - px * PAIRS;
                    va[j] = vb[j] = 0;
                    if (px < g) {
                        ll_load2(xin + (size_t)(p0 + px) * NL + 2 * q, va[j], vb[j]);
                        if ((unsigned)(va[j] >> 32) != want || (unsigned)(vb[j] >> 32) != want) bad |= 1u << px;
                    }
                }
                bad = __reduce_or_sync(kFullMask, bad);
                const int n = bad ? __ffs(bad) - 1 : g;   // the leading pixels that are complete
                if (n > 0) {
#pragma unroll
                    for (int j = 0; j < PER; ++j) {
                        const int f = lane + 32 * j;
                        const int px = f / PAIRS, q = f - px * PAIRS;
                        if (px < n) {
                            uint8_t* dst = sm + L.imp + ((p0 + px) & (kPQ - 1)) * SB + 8 * q;
                            *reinterpret_cast<uint2*>(dst) = make_uint2((uint32_t)va[j], (uint32_t)vb[j]);
                        }
                    }
                    __syncwarp();
                    if (lane == 0) w_st_release_cta(&sctr[0], (unsigned)(p0 + n));
                    p0 += n;
                    spins = 0;
                    nap = 32;
                    continue;
                }
                // nothing new: bounded wait for the band above
                if (sflag[1]) {
                    ok = false;
                    break;
                }
                if ((spins & 63) == 63 && *(volatile int*)a.status != 0) {
                    sflag[1] = 1;
                    ok = false;
                    break;
                }
                if (++spins >= a.spinMax) {
                    if (lane == 0) atomicExch(a.status, (int)LUMEN_ERR_TIMEOUT);
                    sflag[1] = 1;
                    ok = false;
                    break;
                }
                __nanosleep(32);   // the probe saw the epoch: the rest of the pixel is on its way
            }
        }
        if (__syncthreads_or(!ok || sflag[1] != 0)) break;
    }
}

// Eight paths: R/(32/T) row warps and the import warp.
// Register budget: 16-row bands of 8-lane rows are held to three CTAs an SM
// (their shared memory at 1080p allows three) and 24-row bands to two; the
// 16-lane instances keep the compiler's own choice (0), except the widest
// (320 disparities), which is held to one CTA an SM.
template <int KW, int R, int T>
constexpr int pair_min_blocks() {
    return T == 8 ? (R == 16 ? 3 : R == 24 ? 2 : 0) : (KW == 10 ? 1 : 0);
}
template <int KW, bool WRAP, bool FULL, int R, int T>
__global__ void __launch_bounds__((R / (32 / T) + 1) * 32, pair_min_blocks<KW, R, T>()) pair_kernel(PairArgs a) {
    pair_body<KW, WRAP, FULL, R, T, true>(a);
}

// Four paths: row warps only.  The explicit one-CTA-an-SM register budget
// lets the compiler keep more of the next pixel's operands in flight
// (measured faster than the default budget).
template <int KW, bool WRAP, bool FULL, int R, int T>
__global__ void __launch_bounds__(R / (32 / T) * 32, 1) pair4_kernel(PairArgs a) {
    pair_body<KW, WRAP, FULL, R, T, false>(a);
}

}  // namespace lumen

namespace lumen {

// Launch of one instance (the host picks KW, T and R from the padded
// disparity count and the shared memory).  grid == 0: occupancy query only.
template <int KW, int T, int R, bool DIAG = true>
cudaError_t pair_launch_t(const PairArgs& a, bool wrap, bool full, int smem, int grid, cudaStream_t s,
                          int* perSM) {
    constexpr int threads = (R / (32 / T) + (DIAG ? 1 : 0)) * 32;
    void (*k)(PairArgs);
    if constexpr (DIAG)
        k = wrap ? (full ? pair_kernel<KW, true, true, R, T> : pair_kernel<KW, true, false, R, T>)
                 : (full ? pair_kernel<KW, false, true, R, T> : pair_kernel<KW, false, false, R, T>);
    else
        k = wrap ? (full ? pair4_kernel<KW, true, true, R, T> : pair4_kernel<KW, true, false, R, T>)
                 : (full ? pair4_kernel<KW, false, true, R, T> : pair4_kernel<KW, false, false, R, T>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSM, k, threads, smem);
    if (e != cudaSuccess) return e;
    if (grid <= 0) return cudaSuccess;
    k<<<grid, threads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace lumen
