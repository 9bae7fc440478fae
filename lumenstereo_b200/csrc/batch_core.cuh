// batch_core.cuh -- the multi-pair launch core shared by the batched form
// (batch.cu, lumen_sgbm_batch_*) and the served form (server.cu,
// lumen_server_*): per-pair derivation and buffer layout, grouping by kernel
// class, the job descriptors and ticket tables of one persistent sweep launch
// per group, and the enqueue of every kernel of a set of groups.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

struct BatchPair {
    lumen_stereo_params p;
    const uint8_t* left;
    const uint8_t* right;
    int W, H;
    int16_t* out;
    // derived
    int D, Dp, r, cap;
    bool census, diag, wrap, full;
    SgmConsts k;
    int sched, R;  // aggregation schedule (4 or 6) and rows per band of the layout
    int nBands;    // schedule 4: bands per sweep
    int nb0, nb1;  // schedule 6: bands of the row sweeps and of the column sweeps
    // working buffers: base + byte offsets (oAgg, oPartB, oPartC, oPartD: the
    // sweeps' partial volumes, two for schedule 4, four for schedule 6;
    // oRing, oCtr: schedule 4's exchange rings and counters; oXbuf: schedule
    // 6's band-boundary row buffers, 8 paths only)
    uint8_t* base;
    size_t oCost, oAgg, oPartB, oPartC, oPartD, oDispL, oDispR, oAux0, oAux1, oRing, oCtr, oXbuf;
    size_t xbufBytes;
};

struct BatchGroup {
    int Dp;
    bool diag, wrap, full;
    std::vector<int> pairs;  // indices into the pair vector
    int Wmax = 0;
    int Lmax = 0;            // longest sweep row (max of W, H): schedule 6's staging
    int sched = 4;
    WavePlan plan{};         // schedule 4
    PairPlan pplan{};        // schedule 6
    int nTickets = 0;
    int window = 0;                    // ticket distance the oldest unfinished ticket may need running
    size_t jobsOff = 0, tableOff = 0;  // offsets in the descriptor buffer
};

// Validates the pair (the plain call's rules) and derives its constants.
lumen_status batch_pair_init(BatchPair& q, const lumen_stereo_params* p, const uint8_t* d_left,
                             const uint8_t* d_right, int width, int height, int16_t* d_out);
// Lays the pair's working buffers out from byte offset `start` (256-byte
// aligned pieces) for aggregation schedule `sched` (4 or 6) with R rows per
// band; returns the end offset.
size_t batch_pair_layout(BatchPair& q, int sched, int R, size_t start);
// Bytes batch_pair_layout takes for the pair.
size_t batch_pair_bytes(const BatchPair& q, int sched, int R);
// Rows per band a schedule accepts (4: 4, 8, 16; 6: 16, 24, 32) and its default.
bool batch_rows_valid(int sched, int R);
inline int batch_default_rows(int sched) { return sched == 4 ? 8 : 16; }
// Same class: one sweep kernel instance serves both.
bool batch_same_class(const BatchPair& a, const BatchPair& b);
// Groups `idx` by class, largest span first inside a group.
void batch_group_by_class(const std::vector<BatchPair>& pairs, const std::vector<int>& idx,
                          std::vector<BatchGroup>& groups);
// Plans every group for schedule `sched` and writes its job descriptors and
// ticket table into `host` (resized); descriptor offsets go into the groups.
lumen_status batch_describe(const std::vector<BatchPair>& pairs, std::vector<BatchGroup>& groups,
                            int sched, int R, int numSMs, std::vector<uint8_t>& host);
// The three phases of one group: counters and cost volumes, the persistent
// sweep launch, selection and post-processing (each adds its kernels to
// *launches).
lumen_status batch_enqueue_costs(const std::vector<BatchPair>& pairs, const BatchGroup& g, const uint8_t* desc,
                                 const uint32_t* magic, cudaStream_t s, unsigned long long* launches);
lumen_status batch_enqueue_wave(const BatchGroup& g, const uint8_t* desc, int* status, long long spinMax,
                                cudaStream_t s, unsigned long long* launches);
lumen_status batch_enqueue_selects(const std::vector<BatchPair>& pairs, const BatchGroup& g, cudaStream_t s,
                                   unsigned long long* launches);
// Enqueues, group after group, the cost volumes, the sweep launch and the
// selection/post-processing of every pair; `desc` holds the uploaded
// descriptors.  Sweep launches may go to their own stream `agg` (NULL: `s`),
// ordered after the group's cost volumes and before its selections by events
// taken from `evs` (2 per group; NULL when agg is NULL).
lumen_status batch_enqueue_groups(const std::vector<BatchPair>& pairs,
                                  const std::vector<BatchGroup>& groups, const uint8_t* desc,
                                  const uint32_t* magic, int* status, long long spinMax,
                                  cudaStream_t s, cudaStream_t agg, cudaEvent_t* evs,
                                  unsigned long long* launches);

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace lumen
