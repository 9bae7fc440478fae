// api.cu -- host side of the C ABI (include/lumen_sgbm.h).
//
// Restates StereoSGBM (src/sgbm_gpu.cu:100-515) and StereoRectifier
// (src/rectification.cu:259-345) around the B200 kernels: validation in the
// reference's order and with its error categories, device buffers owned by the
// handle and reused across calls (grow-only), every stage enqueued on one
// stream with no host synchronisation between stages (the reference
// synchronises after each stage), and CUDA events for the four timing getters.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <map>
#include <fstream>
#include <sstream>
#include <cstdlib>
#include <vector>

#include "../../include/lumen_sgbm.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace lumen;

namespace {

thread_local std::string g_err;

lumen_status fail(lumen_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define LCU(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(LUMEN_ERR_CUDA, std::string("CUDA error in ") + #call + ": " +       \
                                            cudaGetErrorString(e_));                          \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace

// Records `msg` as this thread's last error (lumen_last_error_string) for
// entry points defined in other translation units.
lumen_status lumen::set_error(lumen_status s, const std::string& msg) { return fail(s, msg); }

struct lumen_sgbm {
    lumen_stereo_params params{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;         // schedule 6: the column sweeps' own launch
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    DevBuf inL, inR, gray[2], pref[2], census[2], cost, agg, dispL, dispR, out, dbgLR, magic;
    DevBuf partB, xring, counters, status;  // sweep schedule: backward partial, exchange rings
    DevBuf partC, partD;                    // schedule 6: the column sweeps' partials
    DevBuf pairBuf;                         // schedule 6: band-boundary row buffers (epoch-tagged words)
    unsigned pairEpoch = 0;                 // epoch of the last schedule-6 launch into pairBuf
    DevBuf trace;                           // lumen_sgbm_debug_trace: band timeline of schedule 4
    int traceOn = 0;
    size_t traceWords = 0;
    int numSMs = 148;
    long long spinMax = 1ll << 22;          // bounded device-side waits
    int stallTest = 0;                      // lumen_sgbm_debug_stall_test
    bool statusPending = false;
    SweepConfig forced{0, 0};               // lumen_sgbm_set_tuning (0 = automatic)
    int forcedNC = -1;                      // lumen_sgbm_set_tuning_columns (-1 = automatic)
    std::map<std::string, std::pair<int, SweepConfig>> tuned;  // key -> (schedule, config)
    int lastSchedule = 0;
    SweepConfig lastConfig{0, 0};
    int magicR = -1;
    float timings[4] = {0, 0, 0, 0};
    unsigned pathOverride = 0;
    int schedule = 0;
    int retain = 0;
    unsigned long long launches = 0;  // kernels enqueued by this handle (all calls)
    bool timingsPending = false;      // events recorded by compute_device, not yet read
    // geometry of the last compute (for debug copies)
    int lastW = 0, lastH = 0, lastD = 0, lastDp = 0, lastMode = -1;
    const uint8_t* lastGray[2] = {nullptr, nullptr};
};

struct lumen_rectifier {
    int W = 0, H = 0;
    bool pre = true;
    DevBuf map[4];
    DevBuf src[2], dst[2];
    cudaStream_t stream = nullptr;
};

// ---------------------------------------------------------------------------
// params (include/stereo/stereo_params.h:57-104)
// ---------------------------------------------------------------------------
extern "C" void lumen_stereo_params_default(lumen_stereo_params* o) {
    if (!o) return;
    o->minDisparity = 0;
    o->maxDisparity = 128;
    o->blockSize = 5;
    o->P1 = 200;
    o->P2 = 800;
    o->preFilterCap = 31;
    o->uniquenessRatio = 10;
    o->disp12MaxDiff = 1;
    o->speckleWindowSize = 100;
    o->speckleRange = 32;
    o->useGPU = 1;
    o->useSharedMemory = 1;
    o->numDirections = 4;
    o->matchingCostMode = 0;
}

extern "C" int lumen_stereo_params_is_valid(const lumen_stereo_params* p) {
    if (!p) return 0;
    if (p->blockSize < 1 || p->blockSize % 2 == 0) return 0;
    if (p->minDisparity < 0) return 0;
    if (p->maxDisparity <= p->minDisparity) return 0;
    if (p->P2 <= p->P1) return 0;
    if (p->uniquenessRatio < 0 || p->uniquenessRatio > 100) return 0;
    return 1;
}

extern "C" void lumen_stereo_params_auto_penalties(lumen_stereo_params* p, int numChannels) {
    if (!p) return;
    p->P1 = 8 * numChannels * p->blockSize * p->blockSize;
    p->P2 = 32 * numChannels * p->blockSize * p->blockSize;
}

extern "C" const char* lumen_last_error_string(void) { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// handle lifetime
// ---------------------------------------------------------------------------
extern "C" lumen_status lumen_sgbm_create(const lumen_stereo_params* params, lumen_sgbm** out) {
    if (!out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_create: out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(LUMEN_ERR_NO_DEVICE, "no CUDA device available");
    lumen_sgbm* h = new lumen_sgbm();
    if (params) h->params = *params;
    else lumen_stereo_params_default(&h->params);
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->numSMs, cudaDevAttrMultiProcessorCount, h->device);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = h->status.ensure(sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->status.p, 0, sizeof(int));
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        lumen_sgbm_destroy(h);
        return fail(LUMEN_ERR_CUDA, std::string("lumen_sgbm_create: ") + cudaGetErrorString(e));
    }
    *out = h;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_destroy(lumen_sgbm* h) {
    if (!h) return LUMEN_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (DevBuf* b : {&h->inL, &h->inR, &h->gray[0], &h->gray[1], &h->pref[0], &h->pref[1],
                      &h->census[0], &h->census[1], &h->cost, &h->agg, &h->dispL, &h->dispR,
                      &h->out, &h->dbgLR, &h->magic, &h->partB, &h->partC, &h->partD, &h->xring,
                      &h->pairBuf, &h->counters, &h->status, &h->trace})
        b->release();
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->evFork) cudaEventDestroy(h->evFork);
    if (h->evJoin) cudaEventDestroy(h->evJoin);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_set_params(lumen_sgbm* h, const lumen_stereo_params* p) {
    if (!h || !p) return fail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_set_params: NULL argument");
    h->params = *p;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_get_params(const lumen_sgbm* h, lumen_stereo_params* out) {
    if (!h || !out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_get_params: NULL argument");
    *out = h->params;
    return LUMEN_OK;
}

// Device-side waits report through a status word; read it once the work is done.
static lumen_status check_status(lumen_sgbm* h) {
    if (!h->statusPending) return LUMEN_OK;
    int st = 0;
    LCU(cudaMemcpy(&st, h->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    h->statusPending = false;
    if (st != 0) {
        cudaMemset(h->status.p, 0, sizeof(int));
        return fail(static_cast<lumen_status>(st),
                    "a bounded device-side wait timed out in the aggregation sweep");
    }
    return LUMEN_OK;
}

static lumen_status read_timings(lumen_sgbm* h) {
    LCU(cudaEventSynchronize(h->ev[4]));
    {
        lumen_status st = check_status(h);
        if (st != LUMEN_OK) return st;
    }
    float t = 0;
    LCU(cudaEventElapsedTime(&t, h->ev[0], h->ev[4]));
    h->timings[0] = t;
    LCU(cudaEventElapsedTime(&t, h->ev[1], h->ev[2]));
    h->timings[1] = t;
    LCU(cudaEventElapsedTime(&t, h->ev[2], h->ev[3]));
    h->timings[2] = t;
    LCU(cudaEventElapsedTime(&t, h->ev[3], h->ev[4]));
    h->timings[3] = t;
    h->timingsPending = false;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_get_timings(lumen_sgbm* h, float out[4]) {
    if (!h || !out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_sgbm_get_timings: NULL argument");
    if (h->timingsPending) {
        lumen_status st = read_timings(h);
        if (st != LUMEN_OK) return st;
    }
    std::memcpy(out, h->timings, sizeof(h->timings));
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_set_wait_limit(lumen_sgbm* h, long long spins) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    if (spins < 0) return fail(LUMEN_ERR_INVALID_ARGUMENT, "wait limit must be >= 0");
    h->spinMax = spins ? spins : (1ll << 22);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_stall_test(lumen_sgbm* h, int enable) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    h->stallTest = enable ? 1 : 0;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_trace(lumen_sgbm* h, int enable) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    h->traceOn = enable ? 1 : 0;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_trace_copy(lumen_sgbm* h, unsigned long long* dst,
                                                    size_t dst_words, size_t* words) {
    if (!h || !words) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    *words = h->traceWords;
    if (!dst || !h->traceWords) return LUMEN_OK;
    if (dst_words < h->traceWords) return fail(LUMEN_ERR_INVALID_ARGUMENT, "destination too small");
    LCU(cudaStreamSynchronize(h->stream));
    LCU(cudaDeviceSynchronize());
    LCU(cudaMemcpy(dst, h->trace.p, h->traceWords * 8, cudaMemcpyDeviceToHost));
    return LUMEN_OK;
}

extern "C" unsigned long long lumen_sgbm_debug_launch_count(const lumen_sgbm* h) {
    return h ? h->launches : 0ull;
}

extern "C" lumen_status lumen_sgbm_debug_set_paths(lumen_sgbm* h, uint32_t mask) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    h->pathOverride = mask & 0xFFu;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_set_schedule(lumen_sgbm* h, int schedule) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    if (!(schedule == 0 || schedule == 1 || schedule == 4 || schedule == 6))
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "schedule must be 0 (automatic), 1, 4 or 6");
    h->schedule = schedule;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_set_tuning(lumen_sgbm* h, int lanes, int warps) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    if (lanes == 0 && warps == 0) {
        h->forced = SweepConfig{0, 0};
        return LUMEN_OK;
    }
    if (!(lanes == 8 || lanes == 16 || lanes == 32) ||
        !(warps == 2 || warps == 4 || warps == 8 || warps == 16 || warps == 24 || warps == 32))
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "lanes must be 8/16/32 and warps 2/4/8/16/24/32");
    h->forced = SweepConfig{lanes, warps};
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_set_tuning_columns(lumen_sgbm* h, int rows) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    if (!(rows == -1 || rows == 0 || rows == 16 || rows == 24 || rows == 32))
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "column rows must be -1 (automatic), 0, 16, 24 or 32");
    h->forcedNC = rows;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_get_tuning(const lumen_sgbm* h, int out[3]) {
    if (!h || !out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    out[0] = h->lastSchedule;
    out[1] = h->lastConfig.T;
    out[2] = h->lastConfig.NW;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_get_tuning_columns(const lumen_sgbm* h, int* rows) {
    if (!h || !rows) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    *rows = h->lastConfig.NC;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_retain(lumen_sgbm* h, int enable) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    h->retain = enable ? 1 : 0;
    return LUMEN_OK;
}

// ---------------------------------------------------------------------------
// validation (src/sgbm_gpu.cu:147-166) and the no-wrap proof
// ---------------------------------------------------------------------------
static lumen_status validate(const lumen_stereo_params& p, const void* l, const void* r, int W,
                             int H, size_t in_stride, int channels) {
    if (!l || !r || W <= 0 || H <= 0)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "Input images are empty");
    if (channels != 1 && channels != 3)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "Input images must have 1 (gray) or 3 (BGR) channels");
    const int D = p.maxDisparity - p.minDisparity;
    if (D < 1)
        return fail(LUMEN_ERR_INVALID_ARGUMENT,
                    "Invalid disparity range: maxDisparity must be greater than minDisparity");
    if (D > LUMEN_MAX_DISPARITY_RANGE)
        return fail(LUMEN_ERR_RANGE_EXCEEDS_LIMIT,
                    "Disparity range (maxDisparity - minDisparity) exceeds GPU limit (" +
                        std::to_string(LUMEN_MAX_DISPARITY_RANGE) + "). Reduce the search range.");
    if (p.minDisparity < 0)
        return fail(LUMEN_ERR_INVALID_ARGUMENT,
                    "minDisparity must be >= 0 (the right-view search would leave the image)");
    if (p.blockSize < 0) return fail(LUMEN_ERR_INVALID_ARGUMENT, "blockSize must be >= 0");
    if (W < 2) return fail(LUMEN_ERR_INVALID_ARGUMENT, "image width must be at least 2");
    if (in_stride && in_stride < (size_t)W * channels)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "in_stride smaller than a row");
    if ((long long)p.maxDisparity * 16 > 32767)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "maxDisparity*16 must fit int16 disparities");
    return LUMEN_OK;
}

static int cost_scale(const lumen_stereo_params& p) {
    if (p.matchingCostMode == 0) return p.blockSize * p.blockSize;          // src/sgbm_gpu.cu:313-314
    return std::max(1, (p.blockSize * p.blockSize * 2 * p.preFilterCap) / 255);  // :316
}

static unsigned path_mask(const lumen_sgbm* h) {
    if (h->pathOverride) return h->pathOverride;
    return h->params.numDirections >= 8 ? 0xFFu : 0x0Fu;  // src/sgbm_gpu.cu:321-359
}

// True when every uint16 quantity of the recurrence provably stays in
// [0, 65535] without wrapping, so packed 32-bit integer arithmetic is exact.
static bool no_wrap(const lumen_stereo_params& p, int cs, int nPaths) {
    if (p.P1 < 0 || cs < 0) return false;
    if (std::abs((long long)p.P2) >= (1ll << 27)) return false;
    const long long cmax = 255ll * cs;
    const long long p2max = std::max<long long>((long long)p.P1 + 1, (long long)p.P2);
    const long long lmax = cmax + p2max;
    if (cmax > 65535) return false;
    if (lmax + p.P1 > 65535) return false;
    if (lmax + p2max > 65535) return false;
    if (lmax * nPaths > 65535) return false;
    return true;
}

// Autotuner key: geometry, disparity range, cost mode, path set, arithmetic mode.
static std::string tune_key(int W, int H, const lumen_stereo_params& p, unsigned mask, bool wrap) {
    std::ostringstream o;
    o << W << "x" << H << ":D" << (p.maxDisparity - p.minDisparity) << ":m" << p.matchingCostMode
      << ":p" << mask << ":w" << (wrap ? 1 : 0);
    return o.str();
}

// ---------------------------------------------------------------------------
// the pipeline (src/sgbm_gpu.cu:197-515)
// ---------------------------------------------------------------------------
static lumen_status run_pipeline(lumen_sgbm* h, const uint8_t* dl, const uint8_t* dr,
                                 size_t pitch, int channels, int W, int H, int16_t* dout,
                                 size_t outPitchElems, cudaStream_t s, bool timed) {
    const lumen_stereo_params& p = h->params;
    const int D = p.maxDisparity - p.minDisparity;
    const int Dp = padded_d(D);
    const size_t N = (size_t)W * H, ND = N * (size_t)Dp;
    const bool census = p.matchingCostMode == 1;
    const uint8_t* gl;
    const uint8_t* gr;
    if (channels == 1 && pitch == (size_t)W) {
        gl = dl;
        gr = dr;
    } else {
        LCU(h->gray[0].ensure(N));
        LCU(h->gray[1].ensure(N));
        launch_stage_gray(dl, dr, pitch, channels, W, H, h->gray[0].as<uint8_t>(),
                          h->gray[1].as<uint8_t>(), s);
        gl = h->gray[0].as<uint8_t>();
        gr = h->gray[1].as<uint8_t>();
    }
    LCU(h->cost.ensure(ND));
    LCU(h->agg.ensure(ND * 2));
    LCU(h->dispL.ensure(N * 2));
    LCU(h->dispR.ensure(N * 2));
    if (h->retain) LCU(h->dbgLR.ensure(N * 2));
    if (timed) LCU(cudaEventRecord(h->ev[1], s));
    unsigned long long nl = (channels == 1 && pitch == (size_t)W) ? 0 : 1;
    // cost volume
    if (census) {
        LCU(h->census[0].ensure(N * 4));
        LCU(h->census[1].ensure(N * 4));
        launch_census(gl, gr, W, H, h->census[0].as<uint32_t>(), h->census[1].as<uint32_t>(), s);
        LCU(launch_census_cost(h->census[0].as<uint32_t>(), h->census[1].as<uint32_t>(), W, H, D, Dp,
                               p.minDisparity, h->cost.as<uint8_t>(), s));
        nl += 2;
    } else {
        const int cap = std::max(1, p.preFilterCap);
        const int r = p.blockSize / 2;
        const int nmagic = (2 * r + 1) * (2 * r + 1) + 1;
        LCU(h->pref[0].ensure(N));
        LCU(h->pref[1].ensure(N));
        if (h->magicR != r) {
            LCU(h->magic.ensure((size_t)nmagic * 4));
            LCU(launch_magic(h->magic.as<uint32_t>(), nmagic, s));
            h->magicR = r;
            nl += 1;
        }
        launch_prefilter(gl, gr, W, H, cap, h->pref[0].as<uint8_t>(), h->pref[1].as<uint8_t>(), s);
        const int wide = (long long)(2 * r + 1) * (2 * r + 1) * 2 * cap > 65535;
        LCU(launch_sad_cost(h->pref[0].as<uint8_t>(), h->pref[1].as<uint8_t>(), W, H, D, Dp,
                            p.minDisparity, r, h->magic.as<uint32_t>(), wide,
                            h->cost.as<uint8_t>(), s));
        nl += 2;
    }
    LCU(cudaGetLastError());
    if (timed) LCU(cudaEventRecord(h->ev[2], s));
    // aggregation
    const unsigned mask = path_mask(h);
    SgmConsts k;
    k.W = W; k.H = H; k.D = D; k.Dp = Dp;
    k.P1 = p.P1; k.P2 = p.P2;
    k.costScale = cost_scale(p);
    k.p1x2 = ((uint32_t)p.P1 & 0xFFFFu) * 0x10001u;
    k.bsub = ((uint32_t)(0xFFFF - p.P1) & 0xFFFFu) * 0x10001u;
    const bool wrap = !no_wrap(p, k.costScale, __builtin_popcount(mask));
    PairView pv{h->cost.as<uint8_t>(), gl, h->agg.as<uint16_t>()};
    const bool sweepable = (mask == 0xFFu || mask == 0x0Fu);
    int sched = h->schedule;
    SweepConfig cfg = h->forced.T ? h->forced : SweepConfig{32, 16};
    bool cfgChosen = h->forced.T != 0;  // pinned or tuned, not a schedule's default
    if (!h->forced.T && sched == 0) {
        auto it = h->tuned.find(tune_key(W, H, p, mask, wrap));
        if (it != h->tuned.end()) {
            sched = it->second.first;
            cfg = it->second.second;
            cfgChosen = true;
        }
    }
    // untuned default: the four lag-free sweeps (schedule 6; with 4 paths one
    // path a sweep), which falls back to schedule 4 where it has no instance
    if (sched == 0) sched = sweepable ? 6 : 1;
    if (sched != 1 && !sweepable) sched = 1;          // single-path debug masks: per-direction kernels
    PairPlan plan6{};
    if (sched == 6) {
        // no instance for this range, or short of device memory for the four
        // partial volumes and the row buffers: schedule 4.  Rows per band and
        // lanes per row: a pinned or tuned configuration when schedule 6 has
        // that instance, else the defaults
        const bool diag = mask == 0xFFu;
        const int R6 = (cfgChosen && (cfg.NW == 16 || cfg.NW == 24 || cfg.NW == 32)) ? cfg.NW : 0;
        const int T6 = cfgChosen ? cfg.T : 0;
        // the column sweeps' own launch: pinned, tuned, or the default (a
        // configuration pinned by lumen_sgbm_set_tuning alone keeps one launch)
        const int Rc6 = !diag                ? 0
                        : h->forcedNC >= 0   ? h->forcedNC
                        : h->forced.T        ? 0
                        : cfgChosen          ? cfg.NC
                                             : kPairDefaultColumnRows;
        bool ok6 = pair_plan(k, wrap, diag, h->numSMs, &plan6, R6, T6, Rc6) == cudaSuccess ||
                   pair_plan(k, wrap, diag, h->numSMs, &plan6, 0, 0, Rc6) == cudaSuccess ||
                   pair_plan(k, wrap, diag, h->numSMs, &plan6) == cudaSuccess;
        if (ok6)
            ok6 = h->partB.ensure(ND * 2) == cudaSuccess && h->partC.ensure(ND * 2) == cudaSuccess &&
                  h->partD.ensure(ND * 2) == cudaSuccess;
        if (ok6 && h->pairBuf.n < plan6.xbufBytes) {
            ok6 = h->pairBuf.ensure(plan6.xbufBytes) == cudaSuccess;
            h->pairEpoch = 0xFFFFFFFFu;                // a new buffer: zeroed before its first use
        }
        if (ok6) ok6 = h->counters.ensure(sizeof(unsigned) * plan6.counterWords) == cudaSuccess;
        if (!ok6) {
            (void)cudaGetLastError();                  // a failed allocation is not a sticky error
            sched = 4;
            if (!h->forced.T) cfgChosen = false;
        }
    }
    WavePlan plan4{};
    // untuned default of the row-band sweeps: 16-row bands, rows as 8-lane
    // teams where the disparity range allows (the best plain configuration
    // measured on 1920x1080 D128; the autotuner refines it per workload)
    if (sched == 4 && !cfgChosen) cfg = SweepConfig{wave_team_exists(Dp, 8) ? 8 : 32, 16};
    bool teamPlanned = false;
    if (sched == 4 && cfg.T != 32 && wave_team_exists(Dp, cfg.T) &&
        (cfg.NW == 8 || cfg.NW == 16 || cfg.NW == 32)) {
        // rows as lane teams of cfg.T lanes (an autotuner candidate)
        if (wave_plan(k, cfg.NW, wrap, mask == 0xFFu, h->numSMs, &plan4, cfg.T) == cudaSuccess)
            teamPlanned = true;
        else
            cfg = SweepConfig{32, cfg.NW};
    }
    if (sched == 4 && !teamPlanned) {
        const int R = (cfg.T == 32 && (cfg.NW == 4 || cfg.NW == 8 || cfg.NW == 16)) ? cfg.NW : 8;
        if (wave_plan(k, R, wrap, mask == 0xFFu, h->numSMs, &plan4) == cudaSuccess ||
            wave_plan(k, 8, wrap, mask == 0xFFu, h->numSMs, &plan4) == cudaSuccess ||
            wave_plan(k, 4, wrap, mask == 0xFFu, h->numSMs, &plan4) == cudaSuccess) {
            cfg = SweepConfig{32, plan4.R};  // lanes per pixel, rows per band
        } else {
            sched = 1;                       // no band fits shared memory: per-direction kernels
        }
    }
    const uint16_t* aggB = nullptr;
    const uint16_t* aggC = nullptr;
    const uint16_t* aggD = nullptr;
    if (sched == 6) {
        LCU(h->partB.ensure(ND * 2));
        LCU(h->partC.ensure(ND * 2));
        LCU(h->partD.ensure(ND * 2));
        LCU(h->counters.ensure(sizeof(unsigned) * plan6.counterWords));
        // every word of the row buffers must carry an epoch below the launch's:
        // zero them when they are new (marked by the epoch at its maximum) and
        // before the epoch would wrap
        unsigned epoch = 0;
        if (plan6.diag) {
            if (h->pairEpoch >= 0xFFFFFFF0u) {
                LCU(cudaMemsetAsync(h->pairBuf.p, 0, h->pairBuf.n, s));
                h->pairEpoch = 0;
            }
            epoch = ++h->pairEpoch;
        }
        uint16_t* const parts[4] = {h->agg.as<uint16_t>(), h->partB.as<uint16_t>(), h->partC.as<uint16_t>(),
                                    h->partD.as<uint16_t>()};
        unsigned long long* trace = nullptr;
        if (h->traceOn) {
            h->traceWords = 4 * ((size_t)plan6.nTickets + plan6.nTicketsC);
            LCU(h->trace.ensure(h->traceWords * 8));
            LCU(cudaMemsetAsync(h->trace.p, 0, h->traceWords * 8, s));
            trace = h->trace.as<unsigned long long>();
        }
        LCU(launch_aggregate_pair(pv, parts, k, wrap, plan6, h->pairBuf.as<unsigned long long>(), epoch,
                                  h->counters.as<unsigned>(), h->status.as<int>(), h->spinMax, s,
                                  h->stallTest, trace, h->stream2, h->evFork, h->evJoin));
        h->statusPending = true;
        nl += 1;
        cfg = SweepConfig{plan6.T, plan6.R, plan6.Rc};
        aggB = parts[1];
        aggC = parts[2];
        aggD = parts[3];
        if (h->retain || select_needs_summed_volume(D, Dp)) {
            for (int i = 1; i < 4; ++i) launch_sum_volumes(parts[0], parts[i], parts[0], ND, s);
            LCU(cudaGetLastError());
            nl += 3;
            aggB = aggC = aggD = nullptr;
        }
    } else if (sched == 4) {
        LCU(h->partB.ensure(ND * 2));
        LCU(h->xring.ensure(plan4.ringBytes));
        LCU(h->counters.ensure(sizeof(unsigned) * plan4.counterWords));
        unsigned long long* trace = nullptr;
        if (h->traceOn) {
            h->traceWords = 4 * 2 * (size_t)plan4.nBands;
            LCU(h->trace.ensure(h->traceWords * 8));
            LCU(cudaMemsetAsync(h->trace.p, 0, h->traceWords * 8, s));
            trace = h->trace.as<unsigned long long>();
        }
        LCU(launch_aggregate_wave(pv, h->partB.as<uint16_t>(), k, wrap, mask == 0xFFu, plan4,
                                  h->xring.as<uint8_t>(), h->counters.as<unsigned>(),
                                  h->status.as<int>(), h->spinMax, s, h->stallTest, trace));
        h->statusPending = true;
        nl += 1;
        aggB = h->partB.as<uint16_t>();
        if (h->retain || select_needs_summed_volume(D, Dp)) {
            launch_sum_volumes(h->agg.as<uint16_t>(), aggB, h->agg.as<uint16_t>(), ND, s);
            LCU(cudaGetLastError());
            nl += 1;
            aggB = nullptr;
        }
    } else {
        LCU(launch_aggregate_per_direction(pv, k, mask, wrap, s));
        nl += __builtin_popcount(mask);
    }
    h->lastSchedule = sched;
    h->lastConfig = sched != 1 ? cfg : SweepConfig{0, 0};
    if (timed) LCU(cudaEventRecord(h->ev[3], s));
    // selection + post-processing
    LCU(launch_select(h->agg.as<uint16_t>(), aggB, wrap, W, H, D, Dp, p.minDisparity,
                      p.uniquenessRatio, h->dispL.as<int16_t>(), h->dispR.as<int16_t>(), s, aggC, aggD));
    const int lr = p.disp12MaxDiff >= 0 ? p.disp12MaxDiff * 16 : -1;
    const int spk = p.speckleWindowSize > 0 ? std::min(p.speckleWindowSize, 25) : 0;
    LCU(launch_post(h->dispL.as<int16_t>(), h->dispR.as<int16_t>(), W, H, lr, spk,
                    p.speckleRange * 16, dout, outPitchElems,
                    h->retain ? h->dbgLR.as<int16_t>() : nullptr, s));
    nl += 2;
    if (timed) LCU(cudaEventRecord(h->ev[4], s));
    h->launches += nl;
    h->lastW = W; h->lastH = H; h->lastD = D; h->lastDp = Dp; h->lastMode = p.matchingCostMode;
    h->lastGray[0] = gl; h->lastGray[1] = gr;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_compute(lumen_sgbm* h, const uint8_t* left,
                                           const uint8_t* right, int width, int height,
                                           size_t in_stride, int channels, int16_t* out,
                                           size_t out_stride) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    lumen_status st = validate(h->params, left, right, width, height, in_stride, channels);
    if (st != LUMEN_OK) return st;
    if (!out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "output buffer is NULL");
    const size_t row = (size_t)width * channels;
    if (!in_stride) in_stride = row;
    if (!out_stride) out_stride = (size_t)width * 2;
    if (out_stride < (size_t)width * 2) return fail(LUMEN_ERR_INVALID_ARGUMENT, "out_stride smaller than a row");
    LCU(cudaSetDevice(h->device));
    const size_t N = (size_t)width * height;
    LCU(h->inL.ensure(row * height));
    LCU(h->inR.ensure(row * height));
    LCU(h->out.ensure(N * 2));
    cudaStream_t s = h->stream;
    LCU(cudaEventRecord(h->ev[0], s));
    LCU(cudaMemcpy2DAsync(h->inL.p, row, left, in_stride, row, height, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpy2DAsync(h->inR.p, row, right, in_stride, row, height, cudaMemcpyHostToDevice, s));
    st = run_pipeline(h, h->inL.as<uint8_t>(), h->inR.as<uint8_t>(), row, channels, width, height,
                      h->out.as<int16_t>(), (size_t)width, s, true);
    if (st != LUMEN_OK) return st;
    LCU(cudaMemcpy2DAsync(out, out_stride, h->out.p, (size_t)width * 2, (size_t)width * 2, height,
                          cudaMemcpyDeviceToHost, s));
    LCU(cudaStreamSynchronize(s));
    return read_timings(h);  // also reports a device-side timeout
}

extern "C" lumen_status lumen_sgbm_compute_device(lumen_sgbm* h, const uint8_t* d_left,
                                                  const uint8_t* d_right, int width, int height,
                                                  size_t in_stride, int channels, int16_t* d_out,
                                                  size_t out_stride, void* stream) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    lumen_status st = validate(h->params, d_left, d_right, width, height, in_stride, channels);
    if (st != LUMEN_OK) return st;
    if (!d_out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "output buffer is NULL");
    const size_t row = (size_t)width * channels;
    if (!in_stride) in_stride = row;
    if (!out_stride) out_stride = (size_t)width * 2;
    if (out_stride < (size_t)width * 2 || out_stride % 2)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "out_stride must be an even byte count >= 2*width");
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the default stream
    LCU(cudaEventRecord(h->ev[0], s));
    st = run_pipeline(h, d_left, d_right, in_stride, channels, width, height, d_out,
                      out_stride / 2, s, true);
    if (st == LUMEN_OK) h->timingsPending = true;
    return st;
}

// Autotuner: every aggregation schedule / sweep configuration runs `repeats`
// times on the caller's device pair; the fastest whole-pipeline device time
// is kept for this workload key (lumen_sgbm_compute_device then uses it).
extern "C" lumen_status lumen_sgbm_autotune(lumen_sgbm* h, const uint8_t* d_left,
                                            const uint8_t* d_right, int width, int height,
                                            size_t in_stride, int channels, int repeats,
                                            char* report, size_t report_bytes) {
    if (!h) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL handle");
    lumen_status st = validate(h->params, d_left, d_right, width, height, in_stride, channels);
    if (st != LUMEN_OK) return st;
    if (repeats < 1) repeats = 1;
    const size_t row = (size_t)width * channels;
    if (!in_stride) in_stride = row;
    LCU(h->out.ensure((size_t)width * height * 2));
    const lumen_stereo_params& p = h->params;
    const int D = p.maxDisparity - p.minDisparity, Dp = padded_d(D);
    const unsigned mask = path_mask(h);
    const bool wrap = !no_wrap(p, cost_scale(p), __builtin_popcount(mask));
    const std::string key = tune_key(width, height, p, mask, wrap);
    std::vector<std::pair<int, SweepConfig>> cands;
    cands.push_back({1, SweepConfig{0, 0}});
    if (mask == 0xFFu || mask == 0x0Fu) {
        int rs[4];
        const int nw = wave_rows_options(Dp, rs, 4);
        for (int i = 0; i < nw; ++i) cands.push_back({4, SweepConfig{32, rs[i]}});
        for (int tl : {8, 16}) {
            if (!wave_team_exists(Dp, tl)) continue;
            cands.push_back({4, SweepConfig{tl, 8}});
            cands.push_back({4, SweepConfig{tl, 16}});
            cands.push_back({4, SweepConfig{tl, 32}});
        }
        // schedule 6 takes `warps` as its rows per band (4 paths: 16 only)
        // (8 paths: all four sweeps in one launch, or the column sweeps in a
        // launch of their own with `NC` rows per band)
        const int t6 = pair_lanes(Dp);
        if (t6) {
            cands.push_back({6, SweepConfig{t6, 16}});
            if (mask == 0xFFu) {
                cands.push_back({6, SweepConfig{t6, 24}});
                cands.push_back({6, SweepConfig{t6, 32}});
                for (int nw : {16, 24})
                    for (int nc : {16, 24, 32})
                        if (nc >= nw) cands.push_back({6, SweepConfig{t6, nw, nc}});
            }
        }
    }
    const SweepConfig savedForced = h->forced;
    const int savedNC = h->forcedNC;
    const int savedSched = h->schedule;
    std::ostringstream rep;
    float bestMs = 1e30f;
    std::pair<int, SweepConfig> best = cands[0];
    for (auto& c : cands) {
        h->schedule = c.first;
        h->forced = c.second;
        h->forcedNC = c.second.NC;
        float acc = 0.f;
        bool ok = true;
        for (int r = 0; r <= repeats; ++r) {  // first run warms up
            LCU(cudaEventRecord(h->ev[0], h->stream));
            st = run_pipeline(h, d_left, d_right, in_stride, channels, width, height,
                              h->out.as<int16_t>(), (size_t)width, h->stream, true);
            if (st != LUMEN_OK) { ok = false; break; }
            LCU(cudaStreamSynchronize(h->stream));
            st = read_timings(h);
            if (st != LUMEN_OK) { ok = false; break; }
            if (r > 0) acc += h->timings[0];
        }
        if (!ok || h->lastSchedule != c.first || h->lastConfig.NC != c.second.NC) continue;
        const float ms = acc / repeats;
        rep << "schedule=" << c.first << " lanes=" << c.second.T << " warps=" << c.second.NW;
        if (c.second.NC) rep << " cols=" << c.second.NC;
        rep << " ms=" << ms << "\n";
        if (ms < bestMs) { bestMs = ms; best = c; }
    }
    h->schedule = savedSched;
    h->forced = savedForced;
    h->forcedNC = savedNC;
    h->tuned[key] = best;
    rep << "best schedule=" << best.first << " lanes=" << best.second.T << " warps=" << best.second.NW;
    if (best.second.NC) rep << " cols=" << best.second.NC;
    rep << " key=" << key << "\n";
    if (report && report_bytes) {
        const std::string r = rep.str();
        std::snprintf(report, report_bytes, "%s", r.c_str());
    }
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_tuning_save(const lumen_sgbm* h, const char* path) {
    if (!h || !path) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    std::ofstream f(path);
    if (!f) return fail(LUMEN_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
    for (auto& kv : h->tuned)
        f << kv.first << " " << kv.second.first << " " << kv.second.second.T << " "
          << kv.second.second.NW << " " << kv.second.second.NC << "\n";
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_tuning_load(lumen_sgbm* h, const char* path) {
    if (!h || !path) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    std::ifstream f(path);
    if (!f) return fail(LUMEN_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
    // key schedule lanes rows [column rows]; entries of retired schedules are skipped
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string key;
        int sched = 0, T = 0, NW = 0, NC = 0;
        if (!(in >> key >> sched >> T >> NW)) continue;
        if (!(in >> NC)) NC = 0;
        if (sched == 1 || sched == 4 || sched == 6) h->tuned[key] = {sched, SweepConfig{T, NW, NC}};
    }
    return LUMEN_OK;
}

extern "C" lumen_status lumen_sgbm_debug_copy(lumen_sgbm* h, int which, void* dst,
                                              size_t dst_bytes) {
    if (!h || !dst) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t N = (size_t)h->lastW * h->lastH;
    if (!N) return fail(LUMEN_ERR_INVALID_ARGUMENT, "no compute has run yet");
    LCU(cudaStreamSynchronize(h->stream));
    LCU(cudaDeviceSynchronize());
    const void* src = nullptr;
    size_t bytes = 0;
    switch (which) {
    case 0: src = h->pref[0].p; bytes = N; break;
    case 1: src = h->pref[1].p; bytes = N; break;
    case 2: src = h->census[0].p; bytes = N * 4; break;
    case 3: src = h->census[1].p; bytes = N * 4; break;
    case 4:
    case 5: {
        const size_t es = which == 4 ? 1 : 2;
        const void* vol = which == 4 ? h->cost.p : h->agg.p;
        const size_t need = N * h->lastD * es;
        if (!vol) return fail(LUMEN_ERR_INVALID_ARGUMENT, "volume not available");
        if (dst_bytes < need) return fail(LUMEN_ERR_INVALID_ARGUMENT, "destination too small");
        LCU(cudaMemcpy2D(dst, h->lastD * es, vol, h->lastDp * es, h->lastD * es, N,
                         cudaMemcpyDeviceToHost));
        return LUMEN_OK;
    }
    case 6: src = h->dispL.p; bytes = N * 2; break;
    case 7: src = h->dispR.p; bytes = N * 2; break;
    case 8:
        if (!h->retain) return fail(LUMEN_ERR_INVALID_ARGUMENT, "enable lumen_sgbm_debug_retain first");
        src = h->dbgLR.p; bytes = N * 2; break;
    case 9: src = h->lastGray[0]; bytes = N; break;
    case 10: src = h->lastGray[1]; bytes = N; break;
    default: return fail(LUMEN_ERR_INVALID_ARGUMENT, "unknown buffer id");
    }
    if (!src) return fail(LUMEN_ERR_INVALID_ARGUMENT, "buffer not produced by the last compute");
    if (dst_bytes < bytes) return fail(LUMEN_ERR_INVALID_ARGUMENT, "destination too small");
    LCU(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return LUMEN_OK;
}

// ---------------------------------------------------------------------------
// rectification (src/rectification.cu:259-411)
// ---------------------------------------------------------------------------
extern "C" lumen_status lumen_rectifier_create(int width, int height, const float* m0x,
                                               const float* m0y, const float* m1x,
                                               const float* m1y, lumen_rectifier** out) {
    if (!out) return fail(LUMEN_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (width <= 0 || height <= 0) return fail(LUMEN_ERR_INVALID_ARGUMENT, "empty image size");
    lumen_rectifier* r = new lumen_rectifier();
    r->W = width;
    r->H = height;
    r->pre = !(m0x && m0y && m1x && m1y);
    cudaError_t e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !r->pre) {
        const float* src[4] = {m0x, m0y, m1x, m1y};
        const size_t bytes = (size_t)width * height * 4;
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
            e = r->map[i].ensure(bytes);
            if (e == cudaSuccess) e = cudaMemcpy(r->map[i].p, src[i], bytes, cudaMemcpyHostToDevice);
        }
    }
    if (e != cudaSuccess) {
        lumen_rectifier_destroy(r);
        return fail(LUMEN_ERR_CUDA, std::string("lumen_rectifier_create: ") + cudaGetErrorString(e));
    }
    *out = r;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_rectifier_destroy(lumen_rectifier* r) {
    if (!r) return LUMEN_OK;
    if (r->stream) cudaStreamSynchronize(r->stream);
    for (auto& b : r->map) b.release();
    for (auto& b : r->src) b.release();
    for (auto& b : r->dst) b.release();
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return LUMEN_OK;
}

extern "C" int lumen_rectifier_is_pre_rectified(const lumen_rectifier* r) { return r ? r->pre : 1; }

extern "C" lumen_status lumen_rectifier_rectify_device(lumen_rectifier* r, const uint8_t* dl,
                                                       const uint8_t* dr, int channels,
                                                       uint8_t* ol, uint8_t* orr, void* stream) {
    if (!r || !dl || !dr || !ol || !orr) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (channels < 1) return fail(LUMEN_ERR_INVALID_ARGUMENT, "channels must be >= 1");
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the default stream
    const size_t n = (size_t)r->W * r->H * channels;
    if (r->pre) {
        LCU(cudaMemcpyAsync(ol, dl, n, cudaMemcpyDeviceToDevice, s));
        LCU(cudaMemcpyAsync(orr, dr, n, cudaMemcpyDeviceToDevice, s));
        return LUMEN_OK;
    }
    launch_remap(dl, dr, r->map[0].as<float>(), r->map[1].as<float>(), r->map[2].as<float>(),
                 r->map[3].as<float>(), ol, orr, r->W, r->H, channels, 2, s);
    LCU(cudaGetLastError());
    return LUMEN_OK;
}

extern "C" lumen_status lumen_rectifier_rectify(lumen_rectifier* r, const uint8_t* left,
                                                const uint8_t* right, int channels,
                                                uint8_t* ol, uint8_t* orr) {
    if (!r || !left || !right || !ol || !orr) return fail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (channels < 1) return fail(LUMEN_ERR_INVALID_ARGUMENT, "channels must be >= 1");
    const size_t n = (size_t)r->W * r->H * channels;
    if (r->pre) {  // clone (src/rectification.cu:291-295)
        std::memcpy(ol, left, n);
        std::memcpy(orr, right, n);
        return LUMEN_OK;
    }
    for (int i = 0; i < 2; ++i) {
        LCU(r->src[i].ensure(n));
        LCU(r->dst[i].ensure(n));
    }
    cudaStream_t s = r->stream;
    LCU(cudaMemcpyAsync(r->src[0].p, left, n, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(r->src[1].p, right, n, cudaMemcpyHostToDevice, s));
    lumen_status st = lumen_rectifier_rectify_device(r, r->src[0].as<uint8_t>(), r->src[1].as<uint8_t>(),
                                                     channels, r->dst[0].as<uint8_t>(),
                                                     r->dst[1].as<uint8_t>(), s);
    if (st != LUMEN_OK) return st;
    LCU(cudaMemcpyAsync(ol, r->dst[0].p, n, cudaMemcpyDeviceToHost, s));
    LCU(cudaMemcpyAsync(orr, r->dst[1].p, n, cudaMemcpyDeviceToHost, s));
    LCU(cudaStreamSynchronize(s));
    return LUMEN_OK;
}

extern "C" lumen_status lumen_remap(const uint8_t* src, const float* mx, const float* my,
                                    uint8_t* dst, int width, int height, int channels) {
    if (!src || !mx || !my || !dst || width <= 0 || height <= 0 || channels < 1)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "invalid remap arguments");
    const size_t n = (size_t)width * height * channels, m = (size_t)width * height * 4;
    DevBuf ds, dd, dx, dy;
    lumen_status st = LUMEN_OK;
    cudaError_t e = ds.ensure(n);
    if (e == cudaSuccess) e = dd.ensure(n);
    if (e == cudaSuccess) e = dx.ensure(m);
    if (e == cudaSuccess) e = dy.ensure(m);
    if (e == cudaSuccess) e = cudaMemcpy(ds.p, src, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dx.p, mx, m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dy.p, my, m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dd.p, 0, n);
    if (e == cudaSuccess) {
        launch_remap(ds.as<uint8_t>(), ds.as<uint8_t>(), dx.as<float>(), dy.as<float>(),
                     dx.as<float>(), dy.as<float>(), dd.as<uint8_t>(), dd.as<uint8_t>(), width,
                     height, channels, 1, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(dst, dd.p, n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(LUMEN_ERR_CUDA, std::string("lumen_remap: ") + cudaGetErrorString(e));
    ds.release(); dd.release(); dx.release(); dy.release();
    return st;
}

extern "C" lumen_status lumen_bgr_to_gray(const uint8_t* bgr, size_t stride, uint8_t* gray,
                                          int width, int height) {
    if (!bgr || !gray || width <= 0 || height <= 0)
        return fail(LUMEN_ERR_INVALID_ARGUMENT, "invalid bgr_to_gray arguments");
    if (!stride) stride = (size_t)width * 3;
    DevBuf ds, dd;
    lumen_status st = LUMEN_OK;
    cudaError_t e = ds.ensure(stride * height);
    if (e == cudaSuccess) e = dd.ensure((size_t)width * height);
    if (e == cudaSuccess) e = cudaMemcpy(ds.p, bgr, stride * height, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_stage_gray(ds.as<uint8_t>(), ds.as<uint8_t>(), stride, 3, width, height,
                          dd.as<uint8_t>(), dd.as<uint8_t>(), 0, 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(gray, dd.p, (size_t)width * height, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(LUMEN_ERR_CUDA, std::string("lumen_bgr_to_gray: ") + cudaGetErrorString(e));
    ds.release(); dd.release();
    return st;
}
