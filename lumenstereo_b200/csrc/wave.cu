// wave.cu -- host side of schedule 4 (lockstep row-band fused sweeps with lane teams,
// wave_kernel.cuh): shared-memory fit, exchange sizing, launch.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "wave_kernel.cuh"
#include "batch_tickets.h"

namespace lumen {

#define LUMEN_WAVE_DECL(KW)                                                                    \
    cudaError_t wave_dispatch_##KW(const WaveArgs& a, int R, int NP, bool wrap, bool full,     \
                                   int smem, int grid, cudaStream_t s, int* perSM);
LUMEN_WAVE_DECL(1)
LUMEN_WAVE_DECL(2)
LUMEN_WAVE_DECL(3)
LUMEN_WAVE_DECL(4)
LUMEN_WAVE_DECL(5)
LUMEN_WAVE_DECL(6)
LUMEN_WAVE_DECL(7)
LUMEN_WAVE_DECL(8)
#define LUMEN_WAVE_TEAM_DECL(KP, T)                                                            \
    cudaError_t wave_dispatch_team_##KP##_##T(const WaveArgs& a, int R, int NP, bool wrap,     \
                                              bool full, int smem, int grid, cudaStream_t s,   \
                                              int* perSM);
LUMEN_WAVE_TEAM_DECL(1, 8)
LUMEN_WAVE_TEAM_DECL(2, 8)
LUMEN_WAVE_TEAM_DECL(1, 16)
LUMEN_WAVE_TEAM_DECL(2, 16)
LUMEN_WAVE_TEAM_DECL(3, 16)
LUMEN_WAVE_TEAM_DECL(4, 16)
LUMEN_WAVE_TEAM_DECL(5, 16)

// lanes per row of the batched launches: the narrowest team that fits the
// padded disparities in a lane's registers
int wave_team_lanes(int Dp) { return Dp <= 128 ? 8 : Dp <= 320 ? 16 : 32; }
bool wave_team_exists(int Dp, int T) { return T == wave_team_lanes(Dp) || (T == 16 && Dp <= 128); }

static cudaError_t dispatch_wave(const WaveArgs& a, int R, int NP, bool wrap, bool full, int smem,
                                 int grid, cudaStream_t s, int* perSM, int T = 32) {
    if (T != 32) {
        if (!wave_team_exists(a.Dp, T) || (R != 8 && R != 16 && R != 32)) return cudaErrorInvalidValue;
        switch (a.Dp / 64 * 100 + T) {
        case 108: return wave_dispatch_team_1_8(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 208: return wave_dispatch_team_2_8(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 116: return wave_dispatch_team_1_16(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 216: return wave_dispatch_team_2_16(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 316: return wave_dispatch_team_3_16(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 416: return wave_dispatch_team_4_16(a, R, NP, wrap, full, smem, grid, s, perSM);
        case 516: return wave_dispatch_team_5_16(a, R, NP, wrap, full, smem, grid, s, perSM);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (a.Dp / 64) {
    case 1: return wave_dispatch_1(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 2: return wave_dispatch_2(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 3: return wave_dispatch_3(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 4: return wave_dispatch_4(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 5: return wave_dispatch_5(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 6: return wave_dispatch_6(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 7: return wave_dispatch_7(a, R, NP, wrap, full, smem, grid, s, perSM);
    case 8: return wave_dispatch_8(a, R, NP, wrap, full, smem, grid, s, perSM);
    default: return cudaErrorInvalidValue;
    }
}

int wave_rows_options(int Dp, int* out, int max) {
    (void)Dp;
    const int opts[] = {8, 4, 16};
    int n = 0;
    for (int o : opts)
        if (n < max) out[n++] = o;
    return n;
}

// Shared-memory fit (largest helper rings) and occupancy of one kernel class
// at a widest image Wmax.
static cudaError_t plan_class(int Wmax, int Dp, int R, bool wrap, bool full, bool diag, int numSMs,
                              WavePlan* plan, int T = 32) {
    // 32-row bands only as lane teams (at most 8 row warps)
    if (R != 4 && R != 8 && R != 16 && !(R == 32 && T != 32)) return cudaErrorInvalidValue;
    const int NP = diag ? 3 : 1;
    int dev = 0, maxSmem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int Q = 0;
    WaveSmem L{};
    for (int q : {16, 8}) {
        L = wave_smem(Wmax, Dp, R, NP, q, q);
        if (L.total <= maxSmem) {
            Q = q;
            break;
        }
    }
    if (!Q) return cudaErrorInvalidConfiguration;
    WaveArgs a{};
    a.Dp = Dp;
    a.Wmax = Wmax;
    a.QI = a.QX = Q;
    int perSM = 0;
    cudaError_t e = dispatch_wave(a, R, NP, wrap, full, L.total, 0, nullptr, &perSM, T);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    plan->T = T;
    plan->R = R;
    plan->Q = Q;
    plan->smem = L.total;
    // capacity; callers clamp to their ticket count
    plan->grid = perSM * numSMs;
    return cudaSuccess;
}

size_t wave_ring_bytes(int nBands, int Dp, bool diag) {
    return 2 * (size_t)nBands * kWK * (size_t)wave_slot_bytes(Dp, diag ? 3 : 1);
}

cudaError_t wave_plan(const SgmConsts& k, int R, bool wrap, bool diag, int numSMs, WavePlan* plan,
                      int T) {
    if (T != 32 && !wave_team_exists(k.Dp, T)) return cudaErrorInvalidValue;
    cudaError_t e = plan_class(k.W, k.Dp, R, wrap, k.D == k.Dp, diag, numSMs, plan, T);
    if (e != cudaSuccess) return e;
    plan->nBands = (k.H + R - 1) / R;
    // tickets alternate the two sweeps.  The oldest unfinished ticket needs
    // the tickets holding the next wave_lookahead_bands(W) bands of its sweep
    // running.
    plan->nTickets = 2 * plan->nBands;
    const int window = 2 * (wave_lookahead_bands(k.W) + 1);
    if (plan->grid < std::min(plan->nTickets, window + 1)) return cudaErrorInvalidConfiguration;
    plan->grid = std::min(plan->nTickets, plan->grid);
    plan->ringBytes = wave_ring_bytes(plan->nBands, k.Dp, diag);
    plan->counterWords = 4 * (size_t)plan->nBands + 32;
    return cudaSuccess;
}

WaveJob wave_job(const PairView& pv, uint16_t* partB, const SgmConsts& k, int R, uint8_t* xring,
                 unsigned* counters) {
    WaveJob j{};
    j.cost = pv.cost;
    j.img = pv.img;
    j.part[0] = pv.agg;
    j.part[1] = partB;
    j.xring = xring;
    j.nBands = (k.H + R - 1) / R;
    j.prod = counters;
    j.cons = counters + 2 * j.nBands;
    j.W = k.W; j.H = k.H; j.D = k.D;
    j.P1 = k.P1; j.P2 = k.P2; j.costScale = k.costScale;
    j.p1x2 = k.p1x2; j.bsub = k.bsub;
    return j;
}

cudaError_t launch_aggregate_wave(const PairView& pv, uint16_t* partB, const SgmConsts& k,
                                  bool wrap, bool diag, const WavePlan& plan, uint8_t* xring,
                                  unsigned* counters, int* status, long long spinMax,
                                  cudaStream_t s, int stallTest, unsigned long long* trace) {
    WaveArgs a{};
    a.job = wave_job(pv, partB, k, plan.R, xring, counters);
    a.jobs = nullptr;
    a.table = nullptr;
    a.nTickets = plan.nTickets;
    a.Wmax = k.W;
    a.ticket = counters + 4 * plan.nBands;
    a.status = status;
    a.Dp = k.Dp;
    a.QI = a.QX = plan.Q;
    a.spinMax = spinMax;
    a.stallTest = stallTest;
    a.trace = trace;
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * plan.counterWords, s);
    if (e != cudaSuccess) return e;
    int dummy = 0;
    return dispatch_wave(a, plan.R, diag ? 3 : 1, wrap, k.D == k.Dp, plan.smem, plan.grid, s, &dummy, plan.T);
}

int wave_lookahead_bands(int W) { return lookahead_bands(W, kWK); }

cudaError_t wave_batch_plan(int Wmax, int Dp, int R, bool wrap, bool full, bool diag, int numSMs,
                            WavePlan* plan, bool teams) {
    // teams where they exist (8 or 16 rows per band) and were asked for, full warps otherwise
    const int T = teams ? wave_team_lanes(Dp) : 32;
    if (T != 32 && (R == 8 || R == 16) &&
        plan_class(Wmax, Dp, R, wrap, full, diag, numSMs, plan, T) == cudaSuccess)
        return cudaSuccess;
    return plan_class(Wmax, Dp, R, wrap, full, diag, numSMs, plan);
}

cudaError_t launch_aggregate_wave_batch(const WaveJob* d_jobs, const uint32_t* d_table, int nTickets,
                                        int window, int Wmax, int Dp, bool wrap, bool full,
                                        bool diag, const WavePlan& plan, unsigned* ticket,
                                        int* status, long long spinMax, cudaStream_t s) {
    // A CTA takes a ticket only while it runs, and the oldest unfinished
    // ticket needs at most the next `window` tickets running (the bands it
    // waits on and the bands whose ring back-pressure it feels): with
    // window + 1 resident CTAs the oldest ticket always completes.
    const int grid = std::min(nTickets, plan.grid);
    if (grid < std::min(nTickets, window + 1)) return cudaErrorInvalidConfiguration;
    WaveArgs a{};
    a.jobs = d_jobs;
    a.table = d_table;
    a.nTickets = nTickets;
    a.Wmax = Wmax;
    a.ticket = ticket;
    a.status = status;
    a.Dp = Dp;
    a.QI = a.QX = plan.Q;
    a.spinMax = spinMax;
    a.stallTest = 0;
    a.trace = nullptr;
    int dummy = 0;
    return dispatch_wave(a, plan.R, diag ? 3 : 1, wrap, full, plan.smem, grid, s, &dummy, plan.T);
}

}  // namespace lumen
