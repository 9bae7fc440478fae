// kernels.cuh -- launchers of the B200 SGBM kernels (host-callable).
#pragma once
#include <string>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"

namespace lumen {

// Records `msg` as the calling thread's last error and returns `s` (api.cu).
lumen_status set_error(lumen_status s, const std::string& msg);

// Number of path lines of direction dir (LR, RL, TB, BT, TLBR, BRTL, TRBL, BLTR).
__host__ __device__ inline int num_lines(int dir, int W, int H) {
    return dir < 2 ? H : (dir < 4 ? W : W + H - 1);
}

void launch_stage_gray(const uint8_t* l, const uint8_t* r, size_t pitch, int channels, int W,
                       int H, uint8_t* gl, uint8_t* gr, cudaStream_t s, int nImages = 2);
void launch_prefilter(const uint8_t* gl, const uint8_t* gr, int W, int H, int cap, uint8_t* pl,
                      uint8_t* pr, cudaStream_t s);
void launch_census(const uint8_t* gl, const uint8_t* gr, int W, int H, uint32_t* cl, uint32_t* cr,
                   cudaStream_t s);
cudaError_t launch_census_cost(const uint32_t* cl, const uint32_t* cr, int W, int H, int D, int Dp,
                               int minD, uint8_t* cost, cudaStream_t s);
size_t sad_cost_smem(int Dp, int r);
// Reciprocal table of the SAD window sizes: m[c] = ceil(2^32 / c), n entries.
cudaError_t launch_magic(uint32_t* m, int n, cudaStream_t s);
cudaError_t launch_sad_cost(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int Dp,
                            int minD, int r, const uint32_t* magic, int wide, uint8_t* cost,
                            cudaStream_t s);

cudaError_t launch_aggregate_per_direction(const PairView& pv, const SgmConsts& k,
                                           unsigned pathMask, bool wrap, cudaStream_t s);

// A fused-sweep configuration: T lanes per pixel (row) and NW rows per band
// (schedule 4) -- the autotuner's unit.
struct SweepConfig {
    int T;
    int NW;
    int NC = 0;   // schedule 6: rows per band of the column sweeps' own launch (0: one launch)
};
// Untuned schedule 6 with 8 paths: the column sweeps in a launch of their own
// with 24-row bands (1920x1080 D128: aggregation 1.90 -> 1.66 ms).
constexpr int kPairDefaultColumnRows = 24;

// ---- schedule 4: lockstep row-band fused sweeps (wave.cu, wave_kernel.cuh) ----
struct WavePlan {
    int R;                 // rows per band
    int Q;                 // import / export ring slots
    int nBands;            // bands per sweep
    int grid;              // CTAs launched (persistent, ticket-scheduled)
    int smem;              // dynamic shared memory per CTA
    int T = 32;            // lanes per row (batched launches: 8 or 16)
    int nTickets = 0;      // tickets of a single-pair launch
    size_t ringBytes;      // exchange rings, both sweeps
    size_t counterWords;   // prod + cons + ticket
};
int wave_rows_options(int Dp, int* out, int max);
// T < 32: rows as teams of T lanes (wave_team_exists(Dp, T) only).
cudaError_t wave_plan(const SgmConsts& k, int R, bool wrap, bool diag, int numSMs, WavePlan* plan,
                      int T = 32);
// the team width of the batched launches for a padded disparity count (32:
// none), and whether a team kernel of T lanes exists for it
int wave_team_lanes(int Dp);
bool wave_team_exists(int Dp, int T);
// Batched form: one launch over the bands of several pairs of one kernel
// class (padded disparity count, path set, arithmetic mode).  d_jobs / d_table
// live in device memory (see wave_kernel.cuh for their layout).
struct WaveJob;
size_t wave_ring_bytes(int nBands, int Dp, bool diag);
// bands below a band that must run for it to finish a row of W pixels
int wave_lookahead_bands(int W);
WaveJob wave_job(const PairView& pv, uint16_t* partB, const SgmConsts& k, int R, uint8_t* xring,
                 unsigned* counters);
// teams: narrow lane teams per row (throughput over step latency: for groups
// with enough pairs to keep the GPU busy)
cudaError_t wave_batch_plan(int Wmax, int Dp, int R, bool wrap, bool full, bool diag, int numSMs,
                            WavePlan* plan, bool teams = false);
cudaError_t launch_aggregate_wave_batch(const WaveJob* d_jobs, const uint32_t* d_table, int nTickets,
                                        int window, int Wmax, int Dp, bool wrap, bool full,
                                        bool diag, const WavePlan& plan, unsigned* ticket,
                                        int* status, long long spinMax, cudaStream_t s);
cudaError_t launch_aggregate_wave(const PairView& pv, uint16_t* partB, const SgmConsts& k,
                                  bool wrap, bool diag, const WavePlan& plan, uint8_t* xring,
                                  unsigned* counters, int* status, long long spinMax,
                                  cudaStream_t s, int stallTest = 0,
                                  unsigned long long* trace = nullptr);

// ---- schedule 6: four lag-free two-path sweeps (pair.cu, pair_kernel.cuh) ----
struct PairPlan {
    int R, T;              // rows per band, lanes per row
    bool diag;             // 8 paths (the diagonals ride along); false: LR, RL, TB, BT alone
    int nb0, nb1;          // bands of the row sweeps, of the column sweeps
    int nTickets;          // 2 * nb0 + 2 * nb1 (split: 2 * nb0, the row sweeps' launch)
    int grid;              // CTAs launched (persistent, ticket-scheduled)
    int smem;              // dynamic shared memory per CTA
    size_t xbufBytes;      // band-boundary row buffers, all sweeps
    size_t counterWords;   // ticket counters (one a launch)
    // Rc > 0 (8 paths): the column sweeps run as a second, concurrent launch
    // with Rc rows per band; its tickets, CTAs and shared memory
    int Rc, nTicketsC, gridC, smemC;
};
// lanes per row of schedule 6 for a padded disparity count (0: no instance)
int pair_lanes(int Dp);
// diag: 8 paths; false: the 4 paths LR, RL, TB, BT (one per sweep, no band
// hand-offs).  R: rows per band, 16, 24 or 32 with diag, 16 without (0: the
// default, 16); T: lanes per row (0 or pair_lanes(Dp)); Rc (diag only): 0
// runs all four sweeps in one launch, 16, 24 or 32 runs the column sweeps as
// a launch of their own with Rc rows per band (the row sweeps keep R).
// cudaErrorInvalidValue: no instance for these disparities / sizes
cudaError_t pair_plan(const SgmConsts& k, bool wrap, bool diag, int numSMs, PairPlan* plan, int R = 0,
                      int T = 0, int Rc = 0);
// Plan of a batched launch of one kernel class: the pairs' longest sweep row
// Lmax sizes the shared memory; nb0/nb1/nTickets/xbufBytes stay 0 (per pair);
// grid is the resident CTA count (the launch takes at most its ticket count).
cudaError_t pair_batch_plan(int Lmax, int Dp, bool wrap, bool full, bool diag, int numSMs, PairPlan* plan,
                            int R = 0);
// Row-buffer bytes of one 8-path pair (R rows per band).
size_t pair_xbuf_bytes(int W, int H, int Dp, int R);
struct PairJob;
// One launch over the bands of many pairs of one class: d_jobs[pairs],
// d_table[nTickets] (pair << 20 | sweep << 18 | band, every band after the
// band before it in its own sweep); every row-buffer word of the pairs holds
// an epoch below `epoch`.
cudaError_t launch_aggregate_pair_batch(const PairJob* d_jobs, const uint32_t* d_table, int nTickets, int Lmax,
                                        int Dp, bool wrap, bool full, const PairPlan& plan, unsigned epoch,
                                        unsigned* ticket, int* status, long long spinMax, cudaStream_t s);
// part[0..3]: the four sweeps' partial volumes (part[0] may be pv.agg).  xbuf:
// the row buffers (plan.xbufBytes), every word of which holds an epoch below
// `epoch` (zero-filled when allocated, then one epoch per launch, increasing).
// With plan.Rc the column sweeps' launch goes to s2, forked from s by evFork
// and joined back by evJoin.
cudaError_t launch_aggregate_pair(const PairView& pv, uint16_t* const part[4], const SgmConsts& k, bool wrap,
                                  const PairPlan& plan, unsigned long long* xbuf, unsigned epoch,
                                  unsigned* counters, int* status, long long spinMax, cudaStream_t s,
                                  int stallTest = 0, unsigned long long* trace = nullptr,
                                  cudaStream_t s2 = nullptr, cudaEvent_t evFork = nullptr,
                                  cudaEvent_t evJoin = nullptr);

// aggB (nullable): second partial volume summed with agg (mod 2^16 when wrap);
// aggC, aggD (nullable, both or neither): two more (schedule 6).
cudaError_t launch_select(const uint16_t* agg, const uint16_t* aggB, bool wrap, int W, int H,
                          int D, int Dp, int minD, int UR, int16_t* dispL, int16_t* dispR,
                          cudaStream_t s, const uint16_t* aggC = nullptr, const uint16_t* aggD = nullptr);
bool select_needs_summed_volume(int D, int Dp);
// dst = a + b (mod 2^16 per element), n uint16 elements (n even).
void launch_sum_volumes(const uint16_t* a, const uint16_t* b, uint16_t* dst, size_t n,
                        cudaStream_t s);
cudaError_t launch_post(const int16_t* dispL, const int16_t* dispR, int W, int H, int lrMaxDiff,
                        int speckleSize, int speckleDiff, int16_t* out, size_t outPitchElems,
                        int16_t* dbgLR, cudaStream_t s);

void launch_remap(const uint8_t* srcL, const uint8_t* srcR, const float* mxL, const float* myL,
                  const float* mxR, const float* myR, uint8_t* dstL, uint8_t* dstR, int W, int H,
                  int channels, int nImages, cudaStream_t s);

}  // namespace lumen
