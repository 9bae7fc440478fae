// pair.cu -- host side of schedule 6 (four lag-free two-path sweeps,
// pair_kernel.cuh): instance choice, shared-memory fit, buffers, launch.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "pair_kernel.cuh"

namespace lumen {

#define LUMEN_PAIR_EXTERN(KW, T, R) \
    extern template cudaError_t pair_launch_t<KW, T, R>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
LUMEN_PAIR_EXTERN(4, 8, 16)
LUMEN_PAIR_EXTERN(8, 8, 16)
LUMEN_PAIR_EXTERN(4, 8, 32)
LUMEN_PAIR_EXTERN(8, 8, 32)
LUMEN_PAIR_EXTERN(6, 16, 16)
LUMEN_PAIR_EXTERN(8, 16, 16)
LUMEN_PAIR_EXTERN(10, 16, 16)
LUMEN_PAIR_EXTERN(6, 16, 32)
LUMEN_PAIR_EXTERN(8, 16, 32)
LUMEN_PAIR_EXTERN(10, 16, 32)
LUMEN_PAIR_EXTERN(4, 8, 24)
LUMEN_PAIR_EXTERN(8, 8, 24)
LUMEN_PAIR_EXTERN(6, 16, 24)
LUMEN_PAIR_EXTERN(8, 16, 24)
LUMEN_PAIR_EXTERN(10, 16, 24)
#define LUMEN_PAIR_EXTERN4(KW, T) \
    extern template cudaError_t pair_launch_t<KW, T, 16, false>(const PairArgs&, bool, bool, int, int, cudaStream_t, int*);
LUMEN_PAIR_EXTERN4(4, 8)
LUMEN_PAIR_EXTERN4(8, 8)
LUMEN_PAIR_EXTERN4(6, 16)
LUMEN_PAIR_EXTERN4(8, 16)
LUMEN_PAIR_EXTERN4(10, 16)
#undef LUMEN_PAIR_EXTERN
#undef LUMEN_PAIR_EXTERN4

// lanes per row for a padded disparity count (0: no instance)
int pair_lanes(int Dp) { return Dp <= 128 ? 8 : Dp <= 320 ? 16 : 0; }

// whether an instance with T lanes per row and R rows per band exists (wider
// teams for the narrow ranges were measured slower on 1080p D128 -- 2.67 and
// 2.73 ms against 2.03 ms with 8 lanes -- and are not built)
static bool pair_instance(int Dp, int T, int R, bool diag) {
    return T == pair_lanes(Dp) && (diag ? (R == 16 || R == 24 || R == 32) : R == 16);
}

static cudaError_t pair_dispatch(const PairArgs& a, int Dp, int R, int T, bool diag, bool wrap, bool full,
                                 int smem, int grid, cudaStream_t s, int* perSM) {
    if (T != pair_lanes(Dp)) return cudaErrorInvalidValue;
    if (!diag) {
        if (R != 16) return cudaErrorInvalidValue;
        switch (Dp) {
        case 64: return pair_launch_t<4, 8, 16, false>(a, wrap, full, smem, grid, s, perSM);
        case 128: return pair_launch_t<8, 8, 16, false>(a, wrap, full, smem, grid, s, perSM);
        case 192: return pair_launch_t<6, 16, 16, false>(a, wrap, full, smem, grid, s, perSM);
        case 256: return pair_launch_t<8, 16, 16, false>(a, wrap, full, smem, grid, s, perSM);
        case 320: return pair_launch_t<10, 16, 16, false>(a, wrap, full, smem, grid, s, perSM);
        default: return cudaErrorInvalidValue;
        }
    }
    if (R == 16) {
        switch (Dp) {
        case 64: return pair_launch_t<4, 8, 16>(a, wrap, full, smem, grid, s, perSM);
        case 128: return pair_launch_t<8, 8, 16>(a, wrap, full, smem, grid, s, perSM);
        case 192: return pair_launch_t<6, 16, 16>(a, wrap, full, smem, grid, s, perSM);
        case 256: return pair_launch_t<8, 16, 16>(a, wrap, full, smem, grid, s, perSM);
        case 320: return pair_launch_t<10, 16, 16>(a, wrap, full, smem, grid, s, perSM);
        default: return cudaErrorInvalidValue;
        }
    }
    if (R == 24) {
        switch (Dp) {
        case 64: return pair_launch_t<4, 8, 24>(a, wrap, full, smem, grid, s, perSM);
        case 128: return pair_launch_t<8, 8, 24>(a, wrap, full, smem, grid, s, perSM);
        case 192: return pair_launch_t<6, 16, 24>(a, wrap, full, smem, grid, s, perSM);
        case 256: return pair_launch_t<8, 16, 24>(a, wrap, full, smem, grid, s, perSM);
        case 320: return pair_launch_t<10, 16, 24>(a, wrap, full, smem, grid, s, perSM);
        default: return cudaErrorInvalidValue;
        }
    }
    if (R == 32) {
        switch (Dp) {
        case 64: return pair_launch_t<4, 8, 32>(a, wrap, full, smem, grid, s, perSM);
        case 128: return pair_launch_t<8, 8, 32>(a, wrap, full, smem, grid, s, perSM);
        case 192: return pair_launch_t<6, 16, 32>(a, wrap, full, smem, grid, s, perSM);
        case 256: return pair_launch_t<8, 16, 32>(a, wrap, full, smem, grid, s, perSM);
        case 320: return pair_launch_t<10, 16, 32>(a, wrap, full, smem, grid, s, perSM);
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t pair_plan(const SgmConsts& k, bool wrap, bool diag, int numSMs, PairPlan* plan, int R, int T, int Rc) {
    if (!pair_lanes(k.Dp)) return cudaErrorInvalidValue;
    if (R == 0) R = 16;
    if (T == 0) T = pair_lanes(k.Dp);
    if (!pair_instance(k.Dp, T, R, diag)) return cudaErrorInvalidValue;
    if (Rc && (!diag || !pair_instance(k.Dp, T, Rc, true))) return cudaErrorInvalidValue;
    PairPlan p{};
    p.R = R;
    p.T = T;
    p.diag = diag;
    p.Rc = Rc;
    p.nb0 = (k.H + R - 1) / R;
    p.nb1 = (k.W + (Rc ? Rc : R) - 1) / (Rc ? Rc : R);
    const bool full = k.D == k.Dp;
    PairArgs dummy{};
    int perSM = 0;
    if (!Rc) {
        p.nTickets = 2 * p.nb0 + 2 * p.nb1;
        p.smem = pair_smem(std::max(k.W, k.H), k.Dp, R).total;
    } else {
        // row sweeps stage rows of W pixels, column sweeps columns of H
        p.nTickets = 2 * p.nb0;
        p.smem = pair_smem(k.W, k.Dp, R).total;
        p.nTicketsC = 2 * p.nb1;
        p.smemC = pair_smem(k.H, k.Dp, Rc).total;
        if (p.smemC > 227 * 1024) return cudaErrorInvalidValue;
        cudaError_t e = pair_dispatch(dummy, k.Dp, Rc, T, true, wrap, full, p.smemC, 0, nullptr, &perSM);
        if (e != cudaSuccess) return e;
        if (perSM < 1) return cudaErrorInvalidConfiguration;
        p.gridC = std::min(p.nTicketsC, perSM * numSMs);
    }
    if (p.smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = pair_dispatch(dummy, k.Dp, R, T, diag, wrap, full, p.smem, 0, nullptr, &perSM);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    p.grid = std::min(p.nTickets, perSM * numSMs);
    // band-boundary rows only when the diagonals cross the bands
    p.xbufBytes = diag ? pair_xbase(3, p.nb1, k.W, k.H, p.nb0, p.nb1) * (size_t)pair_ll_words(k.Dp) * 8 : 0;
    p.counterWords = Rc ? 2 : 1;   // the ticket counter of each launch
    *plan = p;
    return cudaSuccess;
}

cudaError_t pair_batch_plan(int Lmax, int Dp, bool wrap, bool full, bool diag, int numSMs, PairPlan* plan,
                            int R) {
    if (!pair_lanes(Dp)) return cudaErrorInvalidValue;
    if (R == 0) R = 16;
    const int T = pair_lanes(Dp);
    if (!pair_instance(Dp, T, R, diag)) return cudaErrorInvalidValue;
    PairPlan p{};
    p.R = R;
    p.T = T;
    p.diag = diag;
    p.smem = pair_smem(Lmax, Dp, R).total;
    if (p.smem > 227 * 1024) return cudaErrorInvalidValue;
    PairArgs dummy{};
    int perSM = 0;
    cudaError_t e = pair_dispatch(dummy, Dp, R, T, diag, wrap, full, p.smem, 0, nullptr, &perSM);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    p.grid = perSM * numSMs;
    p.counterWords = 1;
    *plan = p;
    return cudaSuccess;
}

size_t pair_xbuf_bytes(int W, int H, int Dp, int R) {
    const int nb0 = (H + R - 1) / R, nb1 = (W + R - 1) / R;
    return pair_xbase(3, nb1, W, H, nb0, nb1) * (size_t)pair_ll_words(Dp) * 8;
}

PairJob pair_job(const PairView& pv, uint16_t* const part[4], const SgmConsts& k, int R,
                 unsigned long long* xbuf) {
    PairJob J{};
    J.cost = pv.cost;
    J.img = pv.img;
    for (int i = 0; i < 4; ++i) J.part[i] = part[i];
    J.xbuf = xbuf;
    J.W = k.W;
    J.H = k.H;
    J.D = k.D;
    J.nb[0] = (k.H + R - 1) / R;
    J.nb[1] = (k.W + R - 1) / R;
    J.P1 = k.P1;
    J.P2 = k.P2;
    J.costScale = k.costScale;
    J.p1x2 = k.p1x2;
    J.bsub = k.bsub;
    return J;
}

cudaError_t launch_aggregate_pair_batch(const PairJob* d_jobs, const uint32_t* d_table, int nTickets, int Lmax,
                                        int Dp, bool wrap, bool full, const PairPlan& plan, unsigned epoch,
                                        unsigned* ticket, int* status, long long spinMax, cudaStream_t s) {
    PairArgs a{};
    a.jobs = d_jobs;
    a.table = d_table;
    a.nTickets = nTickets;
    a.Lmax = Lmax;
    a.ticket = ticket;
    a.status = status;
    a.spinMax = spinMax;
    a.epoch = epoch;
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    int perSM = 0;
    return pair_dispatch(a, Dp, plan.R, plan.T, plan.diag, wrap, full, plan.smem, std::min(plan.grid, nTickets), s,
                         &perSM);
}

cudaError_t launch_aggregate_pair(const PairView& pv, uint16_t* const part[4], const SgmConsts& k, bool wrap,
                                  const PairPlan& plan, unsigned long long* xbuf, unsigned epoch,
                                  unsigned* counters, int* status, long long spinMax, cudaStream_t s,
                                  int stallTest, unsigned long long* trace, cudaStream_t s2,
                                  cudaEvent_t evFork, cudaEvent_t evJoin) {
    PairArgs a{};
    a.job = pair_job(pv, part, k, plan.R, xbuf);
    a.job.nb[1] = plan.nb1;   // the column sweeps' bands (their own height when split)
    a.nTickets = plan.nTickets;
    a.Lmax = std::max(k.W, k.H);
    a.ticket = counters;
    a.status = status;
    a.spinMax = spinMax;
    a.epoch = epoch;
    a.stallTest = stallTest;
    a.trace = trace;
    const bool full = k.D == k.Dp;
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * plan.counterWords, s);
    if (e != cudaSuccess) return e;
    int perSM = 0;
    if (!plan.Rc) return pair_dispatch(a, k.Dp, plan.R, plan.T, plan.diag, wrap, full, plan.smem, plan.grid, s, &perSM);
    if (!s2 || !evFork || !evJoin) return cudaErrorInvalidValue;
    // the row sweeps on s, the column sweeps on s2: the two share only the
    // (disjoint) row buffers and partial volumes, and wait on nothing of each other
    PairArgs ac = a;
    a.sweeps = 1;
    a.Lmax = k.W;
    ac.sweeps = 2;
    ac.nTickets = plan.nTicketsC;
    ac.Lmax = k.H;
    ac.ticket = counters + 1;
    if (trace) ac.trace = trace + 4 * (size_t)plan.nTickets;
    e = cudaEventRecord(evFork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, evFork, 0);
    if (e == cudaSuccess) e = pair_dispatch(a, k.Dp, plan.R, plan.T, true, wrap, full, plan.smem, plan.grid, s, &perSM);
    if (e == cudaSuccess) e = pair_dispatch(ac, k.Dp, plan.Rc, plan.T, true, wrap, full, plan.smemC, plan.gridC, s2, &perSM);
    if (e == cudaSuccess) e = cudaEventRecord(evJoin, s2);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, evJoin, 0);
    return e;
}

}  // namespace lumen
