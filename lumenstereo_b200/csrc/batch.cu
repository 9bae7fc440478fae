// batch.cu -- batched SGBM (lumen_sgbm_batch_*): many stereo pairs per run.
//
// The plain call (lumen_sgbm_compute_device) runs one pair's aggregation
// wavefront, whose span (about W + 2H steps) leaves most of the GPU idle.  A
// batch groups its pairs by kernel class (padded disparity count, path set,
// arithmetic mode, full padding) and runs each group's aggregation as ONE
// persistent launch of the lockstep row-band sweeps over the bands of all its
// pairs (wave_kernel.cuh, tickets in band-major order within chunks), so the
// wavefronts of different pairs fill the GPU together.  Cost volumes and the
// selection run per pair around it.  Buffers come from one pooled device
// allocation sized by a device-memory budget, in two regions that alternate
// between consecutive groups so that groups overlap on the device (one
// group's sweep beside the next one's cost volumes and the previous one's
// selections); with graphs enabled the whole run is captured once into a
// CUDA graph and replayed.  Every pair's output equals lumen_sgbm_compute_device's for the
// same pair bit for bit.
//
// The launch core (batch_pair_*, batch_group_by_class, batch_describe,
// batch_enqueue_groups) is shared with the served form (server.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/lumen_sgbm.h"
#include "batch_core.cuh"
#include "batch_tickets.h"
#include "common.cuh"
#include "kernels.cuh"
#include "pair_kernel.cuh"
#include "wave_kernel.cuh"

namespace lumen {

namespace {

lumen_status bfail(lumen_status s, const std::string& m) { return set_error(s, m); }

// Same rule as the plain call: every uint16 quantity provably stays in range.
bool batch_no_wrap(const lumen_stereo_params& p, int cs, int nPaths) {
    if (p.P1 < 0 || cs < 0) return false;
    if (std::abs((long long)p.P2) >= (1ll << 27)) return false;
    const long long cmax = 255ll * cs;
    const long long p2max = std::max<long long>((long long)p.P1 + 1, (long long)p.P2);
    const long long lmax = cmax + p2max;
    return cmax <= 65535 && lmax + p.P1 <= 65535 && lmax + p2max <= 65535 && lmax * nPaths <= 65535;
}

size_t ctr_bytes(int nBands) { return (4 * (size_t)nBands + 32) * 4; }

}  // namespace

#define BCU(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return bfail(LUMEN_ERR_CUDA, std::string("CUDA error in ") + #call + ": " +       \
                                             cudaGetErrorString(e_));                          \
    } while (0)

lumen_status batch_pair_init(BatchPair& q, const lumen_stereo_params* p, const uint8_t* d_left,
                             const uint8_t* d_right, int width, int height, int16_t* d_out) {
    if (!p) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL parameters");
    if (!d_left || !d_right || width <= 0 || height <= 0)
        return bfail(LUMEN_ERR_INVALID_ARGUMENT, "Input images are empty");
    if (!d_out) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "output buffer is NULL");
    const int D = p->maxDisparity - p->minDisparity;
    if (D < 1)
        return bfail(LUMEN_ERR_INVALID_ARGUMENT,
                     "Invalid disparity range: maxDisparity must be greater than minDisparity");
    if (D > LUMEN_MAX_DISPARITY_RANGE)
        return bfail(LUMEN_ERR_RANGE_EXCEEDS_LIMIT,
                     "Disparity range (maxDisparity - minDisparity) exceeds GPU limit (512). Reduce the search range.");
    if (p->minDisparity < 0) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "minDisparity must be >= 0");
    if (p->blockSize < 0 || p->blockSize > 21) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "blockSize must be in [0, 21]");
    if (width < 2) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "image width must be at least 2");
    if ((long long)p->maxDisparity * 16 > 32767)
        return bfail(LUMEN_ERR_INVALID_ARGUMENT, "maxDisparity*16 must fit int16 disparities");
    q = BatchPair{};
    q.p = *p;
    q.left = d_left;
    q.right = d_right;
    q.W = width;
    q.H = height;
    q.out = d_out;
    q.D = D;
    q.Dp = padded_d(D);
    q.census = p->matchingCostMode == 1;
    q.diag = p->numDirections >= 8;
    q.r = p->blockSize / 2;
    q.cap = std::max(1, p->preFilterCap);
    const int cs = q.census ? std::max(1, (p->blockSize * p->blockSize * 2 * p->preFilterCap) / 255)
                            : p->blockSize * p->blockSize;
    q.wrap = !batch_no_wrap(*p, cs, q.diag ? 8 : 4);
    q.full = q.D == q.Dp;
    q.k.W = width; q.k.H = height; q.k.D = D; q.k.Dp = q.Dp;
    q.k.P1 = p->P1; q.k.P2 = p->P2; q.k.costScale = cs;
    q.k.p1x2 = ((uint32_t)p->P1 & 0xFFFFu) * 0x10001u;
    q.k.bsub = ((uint32_t)(0xFFFF - p->P1) & 0xFFFFu) * 0x10001u;
    return LUMEN_OK;
}

size_t batch_pair_layout(BatchPair& q, int sched, int R, size_t start) {
    const size_t N = (size_t)q.W * q.H, ND = N * q.Dp;
    if (sched == 6 && !q.diag) R = 16;   // the four one-path sweeps have one band height
    q.sched = sched;
    q.R = R;
    q.nBands = (q.H + R - 1) / R;
    q.nb0 = (q.H + R - 1) / R;
    q.nb1 = (q.W + R - 1) / R;
    size_t o = start;
    auto take = [&](size_t n) { const size_t r0 = o; o += align256(n); return r0; };
    q.oCost = take(ND);
    q.oAgg = take(ND * 2);
    q.oPartB = take(ND * 2);
    q.oPartC = q.oPartD = q.oRing = q.oCtr = q.oXbuf = 0;
    q.xbufBytes = 0;
    if (sched == 6) {
        q.oPartC = take(ND * 2);
        q.oPartD = take(ND * 2);
    }
    q.oDispL = take(N * 2);
    q.oDispR = take(N * 2);
    q.oAux0 = take(q.census ? N * 4 : N);
    q.oAux1 = take(q.census ? N * 4 : N);
    if (sched == 6) {
        if (q.diag) {
            q.xbufBytes = pair_xbuf_bytes(q.W, q.H, q.Dp, R);
            q.oXbuf = take(q.xbufBytes);
        }
    } else {
        q.oRing = take(wave_ring_bytes(q.nBands, q.Dp, q.diag));
        q.oCtr = take(ctr_bytes(q.nBands));
    }
    return o;
}

size_t batch_pair_bytes(const BatchPair& q, int sched, int R) {
    BatchPair t = q;
    return batch_pair_layout(t, sched, R, 0);
}

bool batch_rows_valid(int sched, int R) {
    return sched == 4 ? (R == 4 || R == 8 || R == 16) : sched == 6 ? (R == 16 || R == 24 || R == 32) : false;
}

bool batch_same_class(const BatchPair& a, const BatchPair& b) {
    return a.Dp == b.Dp && a.diag == b.diag && a.wrap == b.wrap && a.full == b.full;
}

void batch_group_by_class(const std::vector<BatchPair>& pairs, const std::vector<int>& idx,
                          std::vector<BatchGroup>& groups) {
    std::map<std::tuple<int, bool, bool, bool>, std::vector<int>> cls;
    for (int i : idx) {
        const BatchPair& q = pairs[i];
        cls[std::make_tuple(q.Dp, q.diag, q.wrap, q.full)].push_back(i);
    }
    for (auto& kv : cls) {
        BatchGroup g;
        g.Dp = std::get<0>(kv.first);
        g.diag = std::get<1>(kv.first);
        g.wrap = std::get<2>(kv.first);
        g.full = std::get<3>(kv.first);
        g.pairs = kv.second;
        // longest wavefront span first: the last chunk of the launch, whose
        // latency is the launch's tail, holds the shortest pairs
        std::stable_sort(g.pairs.begin(), g.pairs.end(), [&](int a, int b) {
            return pairs[a].W + 2 * pairs[a].H > pairs[b].W + 2 * pairs[b].H;
        });
        for (int i : g.pairs) {
            g.Wmax = std::max(g.Wmax, pairs[i].W);
            g.Lmax = std::max(g.Lmax, std::max(pairs[i].W, pairs[i].H));
        }
        groups.push_back(g);
    }
}

lumen_status batch_describe(const std::vector<BatchPair>& pairs, std::vector<BatchGroup>& groups,
                            int sched, int R, int numSMs, std::vector<uint8_t>& host) {
    size_t dOff = 0;
    for (BatchGroup& g : groups) {
        g.sched = sched;
        g.nTickets = 0;
        if (sched == 6) {
            // 4 paths: R is 16 (no hand-offs, the band height only groups rows)
            const int Rg = g.diag ? R : 16;
            cudaError_t e = pair_batch_plan(g.Lmax, g.Dp, g.wrap, g.full, g.diag, numSMs, &g.pplan, Rg);
            if (e != cudaSuccess)
                return bfail(LUMEN_ERR_INVALID_ARGUMENT,
                             std::string("batch: no sweep configuration for a group: ") + cudaGetErrorString(e));
            for (int i : g.pairs) {
                if (pairs[i].R != Rg) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "batch: layout and plan disagree");
                g.nTickets += 2 * pairs[i].nb0 + 2 * pairs[i].nb1;
            }
            g.jobsOff = dOff;
            dOff = align256(dOff + sizeof(PairJob) * g.pairs.size());
        } else {
            // a group of several pairs is throughput-bound: lane teams; a pair or
            // two are bound by the wavefront's step latency: full-warp rows
            const bool teams = g.pairs.size() >= 4;
            cudaError_t e = wave_batch_plan(g.Wmax, g.Dp, R, g.wrap, g.full, g.diag, numSMs, &g.plan, teams);
            if (e != cudaSuccess)
                return bfail(LUMEN_ERR_INVALID_ARGUMENT,
                             std::string("batch: no sweep configuration for a group: ") + cudaGetErrorString(e));
            for (int i : g.pairs) g.nTickets += 2 * pairs[i].nBands;
            g.jobsOff = dOff;
            dOff = align256(dOff + sizeof(WaveJob) * g.pairs.size());
        }
        g.tableOff = dOff;
        dOff = align256(dOff + sizeof(uint32_t) * (size_t)g.nTickets + 4);  // + the ticket counter
    }
    host.assign(dOff, 0);
    for (BatchGroup& g : groups) {
        uint32_t* table = reinterpret_cast<uint32_t*>(host.data() + g.tableOff);
        if (sched == 6) {
            PairJob* jobs = reinterpret_cast<PairJob*>(host.data() + g.jobsOff);
            for (int j = 0; j < (int)g.pairs.size(); ++j) {
                const BatchPair& q = pairs[g.pairs[j]];
                PairView pv{reinterpret_cast<const uint8_t*>(q.base + q.oCost), q.left, nullptr};
                uint16_t* const part[4] = {reinterpret_cast<uint16_t*>(q.base + q.oAgg),
                                           reinterpret_cast<uint16_t*>(q.base + q.oPartB),
                                           reinterpret_cast<uint16_t*>(q.base + q.oPartC),
                                           reinterpret_cast<uint16_t*>(q.base + q.oPartD)};
                jobs[j] = pair_job(pv, part, q.k, q.R,
                                   q.diag ? reinterpret_cast<unsigned long long*>(q.base + q.oXbuf) : nullptr);
            }
            // band-major over the (pair, sweep) chains: every chain's band b comes
            // one round after its band b-1, so a band waits only on an earlier
            // ticket, and all chains start at once
            int maxB = 0;
            for (int i : g.pairs) maxB = std::max(maxB, std::max(pairs[i].nb0, pairs[i].nb1));
            size_t n = 0;
            for (int b = 0; b < maxB; ++b)
                for (int j = 0; j < (int)g.pairs.size(); ++j) {
                    const BatchPair& q = pairs[g.pairs[j]];
                    for (int sw = 0; sw < 4; ++sw)
                        if (b < (sw < 2 ? q.nb0 : q.nb1))
                            table[n++] = (uint32_t)j << 20 | (uint32_t)sw << 18 | (uint32_t)b;
                }
            if ((int)n != g.nTickets) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "batch: ticket table size");
            g.window = 0;
            continue;
        }
        WaveJob* jobs = reinterpret_cast<WaveJob*>(host.data() + g.jobsOff);
        for (int j = 0; j < (int)g.pairs.size(); ++j) {
            const BatchPair& q = pairs[g.pairs[j]];
            PairView pv{reinterpret_cast<const uint8_t*>(q.base + q.oCost), q.left,
                        reinterpret_cast<uint16_t*>(q.base + q.oAgg)};
            jobs[j] = wave_job(pv, reinterpret_cast<uint16_t*>(q.base + q.oPartB), q.k, R, q.base + q.oRing,
                               reinterpret_cast<unsigned*>(q.base + q.oCtr));
        }
        std::vector<TicketPair> tp(g.pairs.size());
        for (int j = 0; j < (int)g.pairs.size(); ++j) tp[j] = TicketPair{pairs[g.pairs[j]].W, pairs[g.pairs[j]].nBands};
        std::vector<uint32_t> tickets;
        g.window = build_ticket_table(tp, g.plan.grid, kWK, tickets);
        if (g.window < 0)
            return bfail(LUMEN_ERR_INVALID_ARGUMENT, "batch: a pair is too wide for the resident sweep CTAs");
        std::copy(tickets.begin(), tickets.end(), table);
    }
    return LUMEN_OK;
}

lumen_status batch_enqueue_costs(const std::vector<BatchPair>& pairs, const BatchGroup& g, const uint8_t* desc,
                                 const uint32_t* magic, cudaStream_t s, unsigned long long* launches) {
    // schedule 4: the counters of the group's pairs; schedule 6: the row
    // buffers (every word below the launch's epoch, 1); the group's ticket
    for (int i : g.pairs) {
        const BatchPair& q = pairs[i];
        if (g.sched == 6) {
            if (q.xbufBytes) BCU(cudaMemsetAsync(q.base + q.oXbuf, 0, q.xbufBytes, s));
        } else {
            BCU(cudaMemsetAsync(q.base + q.oCtr, 0, ctr_bytes(q.nBands), s));
        }
    }
    unsigned* ticket = reinterpret_cast<unsigned*>(const_cast<uint8_t*>(desc) + g.tableOff +
                                                   sizeof(uint32_t) * (size_t)g.nTickets);
    BCU(cudaMemsetAsync(ticket, 0, 4, s));
    for (int i : g.pairs) {
        const BatchPair& q = pairs[i];
        uint8_t* cost = q.base + q.oCost;
        if (q.census) {
            uint32_t* c0 = reinterpret_cast<uint32_t*>(q.base + q.oAux0);
            uint32_t* c1 = reinterpret_cast<uint32_t*>(q.base + q.oAux1);
            launch_census(q.left, q.right, q.W, q.H, c0, c1, s);
            BCU(launch_census_cost(c0, c1, q.W, q.H, q.D, q.Dp, q.p.minDisparity, cost, s));
        } else {
            uint8_t* p0 = q.base + q.oAux0;
            uint8_t* p1 = q.base + q.oAux1;
            launch_prefilter(q.left, q.right, q.W, q.H, q.cap, p0, p1, s);
            const int wide = (long long)(2 * q.r + 1) * (2 * q.r + 1) * 2 * q.cap > 65535;
            BCU(launch_sad_cost(p0, p1, q.W, q.H, q.D, q.Dp, q.p.minDisparity, q.r, magic, wide, cost, s));
        }
        *launches += 2;
    }
    return LUMEN_OK;
}

lumen_status batch_enqueue_wave(const BatchGroup& g, const uint8_t* desc, int* status, long long spinMax,
                                cudaStream_t s, unsigned long long* launches) {
    unsigned* ticket = reinterpret_cast<unsigned*>(const_cast<uint8_t*>(desc) + g.tableOff +
                                                   sizeof(uint32_t) * (size_t)g.nTickets);
    if (g.sched == 6) {
        BCU(launch_aggregate_pair_batch(reinterpret_cast<const PairJob*>(desc + g.jobsOff),
                                        reinterpret_cast<const uint32_t*>(desc + g.tableOff), g.nTickets, g.Lmax,
                                        g.Dp, g.wrap, g.full, g.pplan, 1u, ticket, status, spinMax, s));
        *launches += 1;
        return LUMEN_OK;
    }
    BCU(launch_aggregate_wave_batch(reinterpret_cast<const WaveJob*>(desc + g.jobsOff),
                                    reinterpret_cast<const uint32_t*>(desc + g.tableOff), g.nTickets, g.window,
                                    g.Wmax, g.Dp, g.wrap, g.full, g.diag, g.plan, ticket, status, spinMax, s));
    *launches += 1;
    return LUMEN_OK;
}

lumen_status batch_enqueue_selects(const std::vector<BatchPair>& pairs, const BatchGroup& g, cudaStream_t s,
                                   unsigned long long* launches) {
    for (int i : g.pairs) {
        const BatchPair& q = pairs[i];
        int16_t* dl = reinterpret_cast<int16_t*>(q.base + q.oDispL);
        int16_t* dr = reinterpret_cast<int16_t*>(q.base + q.oDispR);
        uint16_t* agg = reinterpret_cast<uint16_t*>(q.base + q.oAgg);
        uint16_t* pb = reinterpret_cast<uint16_t*>(q.base + q.oPartB);
        uint16_t* pc = nullptr;
        uint16_t* pd = nullptr;
        if (g.sched == 6) {
            pc = reinterpret_cast<uint16_t*>(q.base + q.oPartC);
            pd = reinterpret_cast<uint16_t*>(q.base + q.oPartD);
        }
        BCU(launch_select(agg, pb, q.wrap, q.W, q.H, q.D, q.Dp, q.p.minDisparity, q.p.uniquenessRatio, dl, dr, s,
                          pc, pd));
        const int lr = q.p.disp12MaxDiff >= 0 ? q.p.disp12MaxDiff * 16 : -1;
        const int spk = q.p.speckleWindowSize > 0 ? std::min(q.p.speckleWindowSize, 25) : 0;
        BCU(launch_post(dl, dr, q.W, q.H, lr, spk, q.p.speckleRange * 16, q.out, (size_t)q.W, nullptr, s));
        *launches += 2;
    }
    return LUMEN_OK;
}

lumen_status batch_enqueue_groups(const std::vector<BatchPair>& pairs,
                                  const std::vector<BatchGroup>& groups, const uint8_t* desc,
                                  const uint32_t* magic, int* status, long long spinMax,
                                  cudaStream_t s, cudaStream_t agg, cudaEvent_t* evs,
                                  unsigned long long* launches) {
    unsigned long long nl = 0;
    int gi = 0;
    for (const BatchGroup& g : groups) {
        lumen_status st = batch_enqueue_costs(pairs, g, desc, magic, s, &nl);
        if (st != LUMEN_OK) return st;
        // one aggregation launch over all bands of the group
        cudaStream_t as = s;
        if (agg) {
            BCU(cudaEventRecord(evs[2 * gi], s));
            BCU(cudaStreamWaitEvent(agg, evs[2 * gi], 0));
            as = agg;
        }
        st = batch_enqueue_wave(g, desc, status, spinMax, as, &nl);
        if (st != LUMEN_OK) return st;
        if (agg) {
            BCU(cudaEventRecord(evs[2 * gi + 1], agg));
            BCU(cudaStreamWaitEvent(s, evs[2 * gi + 1], 0));
        }
        st = batch_enqueue_selects(pairs, g, s, &nl);
        if (st != LUMEN_OK) return st;
        ++gi;
    }
    if (launches) *launches = nl;
    return LUMEN_OK;
}

}  // namespace lumen

using namespace lumen;

struct lumen_sgbm_batch {
    std::vector<BatchPair> pairs;
    std::vector<BatchGroup> groups;
    bool planned = false;
    int sched = 0;      // aggregation schedule: 4, 6 (0: 6)
    int rows = 0;       // rows per band (0: the schedule's default)
    int useGraph = 0;
    size_t budget = 80ull << 30;
    int numSMs = 148;
    long long spinMax = 1ll << 22;
    void* pool = nullptr;
    size_t poolBytes = 0;
    void* desc = nullptr;  // WaveJob arrays and ticket tables of all groups
    size_t descBytes = 0;
    uint32_t* magic = nullptr;
    int* status = nullptr;
    cudaStream_t capStream = nullptr;
    // overlapped runs: sweeps on aggS, at the highest priority, selections on
    // selS, cost volumes on the caller's stream
    bool overlap = false;
    cudaStream_t aggS = nullptr, selS = nullptr;
    std::vector<cudaEvent_t> evs;  // fork, 2 joins, then 3 per group
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;  // kernels per run
};

static void batch_release(lumen_sgbm_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    if (b->pool) cudaFree(b->pool);
    if (b->desc) cudaFree(b->desc);
    for (cudaEvent_t e : b->evs) cudaEventDestroy(e);
    b->evs.clear();
    b->overlap = false;
    b->pool = b->desc = nullptr;
    b->poolBytes = b->descBytes = 0;
    b->planned = false;
}

// Buffers, groups, job descriptors and ticket tables for the current pairs.
// Each class is cut into groups whose buffers fit a cap.  Overlapped runs lay
// the groups out alternately in two regions of the pool (even groups in the
// first, odd in the second), so that one group's sweep runs beside the next
// group's cost volumes and the previous group's selections; a group reuses
// its region once the group two before it has been selected.  The cap is the
// budget when the two largest alternate groups fit it together, else half the
// budget.  When even that fails (a single pair above half the budget), the
// groups run one after the other in one region of budget bytes.
static lumen_status batch_plan(lumen_sgbm_batch* b) {
    batch_release(b);
    const int sched = b->sched ? b->sched : 6;
    const int R = b->rows ? b->rows : batch_default_rows(sched);
    if (!batch_rows_valid(sched, R))
        return bfail(LUMEN_ERR_INVALID_ARGUMENT, "batch: rows per band must be 4, 8 or 16 with schedule 4, "
                                                 "16, 24 or 32 with schedule 6");
    std::vector<int> all(b->pairs.size());
    for (int i = 0; i < (int)all.size(); ++i) all[i] = i;
    std::vector<BatchGroup> classes;
    batch_group_by_class(b->pairs, all, classes);
    std::vector<size_t> gbytes;
    bool tooBig = false;
    auto cut = [&](size_t cap) {
        b->groups.clear();
        gbytes.clear();
        tooBig = false;
        for (const BatchGroup& c : classes) {
            BatchGroup g = c;
            g.pairs.clear();
            g.Wmax = 0;
            size_t bytes = 0;
            auto flush = [&]() {
                if (!g.pairs.empty()) {
                    b->groups.push_back(g);
                    gbytes.push_back(bytes);
                }
                g.pairs.clear();
                g.Wmax = 0;
                bytes = 0;
            };
            for (int i : c.pairs) {
                const size_t need = batch_pair_bytes(b->pairs[i], sched, R);
                if (need > cap) tooBig = true;
                if (!g.pairs.empty() && bytes + need > cap) flush();
                bytes += need;
                g.pairs.push_back(i);
                g.Wmax = std::max(g.Wmax, b->pairs[i].W);
            }
            flush();
        }
    };
    auto regions = [&](size_t* even, size_t* odd) {
        *even = *odd = 0;
        for (size_t gi = 0; gi < gbytes.size(); ++gi) {
            size_t& r = gi % 2 ? *odd : *even;
            r = std::max(r, gbytes[gi]);
        }
    };
    cut(b->budget);
    if (tooBig) return bfail(LUMEN_ERR_OUT_OF_BUDGET, "batch: one pair needs more device memory than the budget");
    size_t even = 0, odd = 0;
    regions(&even, &odd);
    if (b->groups.size() > 1 && even + odd > b->budget) {
        cut(b->budget / 2);
        regions(&even, &odd);
        if (tooBig) {  // no two groups fit side by side: one region, groups in turn
            cut(b->budget);
            regions(&even, &odd);
            odd = 0;
        }
    }
    b->overlap = b->groups.size() > 1 && odd > 0;
    size_t poolNeed = 0;
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        size_t o = b->overlap && gi % 2 ? even : 0;
        for (int i : b->groups[gi].pairs) o = batch_pair_layout(b->pairs[i], sched, R, o);
        poolNeed = std::max(poolNeed, o);
    }
    if (b->overlap) {
        b->evs.resize(3 + 3 * b->groups.size(), nullptr);
        for (cudaEvent_t& e : b->evs) BCU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    BCU(cudaMalloc(&b->pool, std::max<size_t>(poolNeed, 256)));
    b->poolBytes = poolNeed;
    for (BatchPair& q : b->pairs) q.base = static_cast<uint8_t*>(b->pool);
    std::vector<uint8_t> host;
    lumen_status st = batch_describe(b->pairs, b->groups, sched, R, b->numSMs, host);
    if (st != LUMEN_OK) return st;
    BCU(cudaMalloc(&b->desc, std::max<size_t>(host.size(), 256)));
    b->descBytes = host.size();
    BCU(cudaMemcpy(b->desc, host.data(), host.size(), cudaMemcpyHostToDevice));
    b->planned = true;
    return LUMEN_OK;
}

static lumen_status batch_enqueue(lumen_sgbm_batch* b, cudaStream_t s) {
    unsigned long long nl = 0;
    const uint8_t* desc = static_cast<const uint8_t*>(b->desc);
    if (!b->overlap) {
        lumen_status st = batch_enqueue_groups(b->pairs, b->groups, desc, b->magic, b->status, b->spinMax, s,
                                               nullptr, nullptr, &nl);
        b->launches = nl;
        return st;
    }
    // fork the sweep and selection streams off `s` (inside a capture too)
    cudaEvent_t* ev = b->evs.data();
    BCU(cudaEventRecord(ev[0], s));
    BCU(cudaStreamWaitEvent(b->aggS, ev[0], 0));
    BCU(cudaStreamWaitEvent(b->selS, ev[0], 0));
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const BatchGroup& g = b->groups[gi];
        cudaEvent_t costsDone = ev[3 + 3 * gi], sweepDone = ev[4 + 3 * gi], selDone = ev[5 + 3 * gi];
        if (gi >= 2) BCU(cudaStreamWaitEvent(s, ev[5 + 3 * (gi - 2)], 0));  // its region is free again
        lumen_status st = batch_enqueue_costs(b->pairs, g, desc, b->magic, s, &nl);
        if (st != LUMEN_OK) return st;
        BCU(cudaEventRecord(costsDone, s));
        BCU(cudaStreamWaitEvent(b->aggS, costsDone, 0));
        st = batch_enqueue_wave(g, desc, b->status, b->spinMax, b->aggS, &nl);
        if (st != LUMEN_OK) return st;
        BCU(cudaEventRecord(sweepDone, b->aggS));
        BCU(cudaStreamWaitEvent(b->selS, sweepDone, 0));
        st = batch_enqueue_selects(b->pairs, g, b->selS, &nl);
        if (st != LUMEN_OK) return st;
        BCU(cudaEventRecord(selDone, b->selS));
    }
    BCU(cudaEventRecord(ev[1], b->aggS));
    BCU(cudaEventRecord(ev[2], b->selS));
    BCU(cudaStreamWaitEvent(s, ev[1], 0));
    BCU(cudaStreamWaitEvent(s, ev[2], 0));
    b->launches = nl;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_create(lumen_sgbm_batch** out) {
    if (!out) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_batch_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return bfail(LUMEN_ERR_NO_DEVICE, "no CUDA device available");
    lumen_sgbm_batch* b = new lumen_sgbm_batch();
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaMalloc(&b->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->status, 0, sizeof(int));
    // reciprocal table for every SAD window up to 21x21 (blockSize <= 21)
    if (e == cudaSuccess) e = cudaMalloc(&b->magic, 443 * sizeof(uint32_t));
    if (e == cudaSuccess) e = launch_magic(b->magic, 443, 0);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capStream, cudaStreamNonBlocking);
    int prLeast = 0, prGreatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
    // sweeps first: their CTAs wait on one another, the other kernels do not
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->aggS, cudaStreamNonBlocking, prGreatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->selS, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        lumen_sgbm_batch_destroy(b);
        return bfail(LUMEN_ERR_CUDA, std::string("lumen_sgbm_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_destroy(lumen_sgbm_batch* b) {
    if (!b) return LUMEN_OK;
    cudaDeviceSynchronize();
    batch_release(b);
    if (b->status) cudaFree(b->status);
    if (b->magic) cudaFree(b->magic);
    if (b->capStream) cudaStreamDestroy(b->capStream);
    if (b->aggS) cudaStreamDestroy(b->aggS);
    if (b->selS) cudaStreamDestroy(b->selS);
    delete b;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_add(lumen_sgbm_batch* b, const lumen_stereo_params* p,
                                             const uint8_t* d_left, const uint8_t* d_right, int width,
                                             int height, int16_t* d_out) {
    if (!b || !p) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_batch_add: NULL argument");
    if (b->pairs.size() >= 4095) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "a batch holds at most 4095 pairs");
    BatchPair q;
    lumen_status st = batch_pair_init(q, p, d_left, d_right, width, height, d_out);
    if (st != LUMEN_OK) return st;
    b->pairs.push_back(q);
    b->planned = false;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_clear(lumen_sgbm_batch* b) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    cudaDeviceSynchronize();
    b->pairs.clear();
    batch_release(b);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_set_options(lumen_sgbm_batch* b, int rows_per_band, int use_graph,
                                                     size_t device_budget_bytes) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    if (rows_per_band != 0 && !batch_rows_valid(4, rows_per_band) && !batch_rows_valid(6, rows_per_band))
        return bfail(LUMEN_ERR_INVALID_ARGUMENT, "rows_per_band must be 0, 4, 8, 16, 24 or 32");
    cudaDeviceSynchronize();
    b->rows = rows_per_band;
    b->useGraph = use_graph ? 1 : 0;
    if (device_budget_bytes) b->budget = device_budget_bytes;
    batch_release(b);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_run(lumen_sgbm_batch* b, void* stream) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    if (b->pairs.empty()) return LUMEN_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!b->planned) {
        lumen_status st = batch_plan(b);
        if (st != LUMEN_OK) return st;
    }
    if (!b->useGraph) return batch_enqueue(b, s);
    if (!b->exec) {
        BCU(cudaStreamBeginCapture(b->capStream, cudaStreamCaptureModeThreadLocal));
        lumen_status st = batch_enqueue(b, b->capStream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->capStream, &g);
        if (st != LUMEN_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        BCU(e);
        b->graph = g;
        BCU(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    BCU(cudaGraphLaunch(b->exec, s));
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_sync(lumen_sgbm_batch* b, void* stream) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    BCU(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    int st = 0;
    BCU(cudaMemcpy(&st, b->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) {
        cudaMemset(b->status, 0, sizeof(int));
        return bfail(static_cast<lumen_status>(st), "a bounded device-side wait timed out in a batched sweep");
    }
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_autotune(lumen_sgbm_batch* b, void* stream, int repeats,
                                                  int* best_rows, float* best_ms) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    if (b->pairs.empty()) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "empty batch");
    if (repeats < 1) repeats = 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCU(cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        return bfail(LUMEN_ERR_CUDA, "batch autotune: event creation failed");
    }
    const int savedGraph = b->useGraph;
    int bestR = 0, bestS = 0;
    float bestMs = 0.f;
    lumen_status st = LUMEN_OK;
    // the schedule pinned by lumen_sgbm_batch_set_schedule, else both
    std::vector<std::pair<int, int>> cands;
    for (int sc : {6, 4})
        if (!b->sched || b->sched == sc)
            for (int R : (sc == 4 ? std::vector<int>{4, 8, 16} : std::vector<int>{16, 24, 32}))
                cands.push_back({sc, R});
    const int savedSched = b->sched;
    for (auto [sc, R] : cands) {
        cudaStreamSynchronize(s);
        batch_release(b);
        b->sched = sc;
        b->rows = R;
        b->useGraph = 0;
        st = lumen_sgbm_batch_run(b, stream);  // plans, warms up
        if (st == LUMEN_OK) st = lumen_sgbm_batch_sync(b, stream);
        if (st != LUMEN_OK) break;
        cudaEventRecord(e0, s);
        for (int i = 0; i < repeats && st == LUMEN_OK; ++i) st = lumen_sgbm_batch_run(b, stream);
        cudaEventRecord(e1, s);
        if (st == LUMEN_OK) st = lumen_sgbm_batch_sync(b, stream);
        if (st != LUMEN_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)repeats;
        if (!bestR || ms < bestMs) {
            bestR = R;
            bestS = sc;
            bestMs = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(s);
    batch_release(b);
    b->useGraph = savedGraph;
    if (st != LUMEN_OK) {
        b->sched = savedSched;
        return st;
    }
    b->sched = bestS;  // the next run plans (and captures) with them
    b->rows = bestR;
    if (best_rows) *best_rows = bestR;
    if (best_ms) *best_ms = bestMs;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_set_schedule(lumen_sgbm_batch* b, int schedule) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    if (schedule != 0 && schedule != 4 && schedule != 6)
        return bfail(LUMEN_ERR_INVALID_ARGUMENT, "batch schedule must be 0 (automatic), 4 or 6");
    cudaDeviceSynchronize();
    b->sched = schedule;
    batch_release(b);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_config(const lumen_sgbm_batch* b, int* schedule, int* rows_per_band) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    const int sc = b->sched ? b->sched : 6;
    if (schedule) *schedule = sc;
    if (rows_per_band) *rows_per_band = b->rows ? b->rows : batch_default_rows(sc);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_batch_info(const lumen_sgbm_batch* b, size_t* device_bytes,
                                              int* groups, unsigned long long* launches) {
    if (!b) return bfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL batch");
    if (device_bytes) *device_bytes = b->poolBytes + b->descBytes;
    if (groups) *groups = (int)b->groups.size();
    if (launches) *launches = b->launches;
    return LUMEN_OK;
}
