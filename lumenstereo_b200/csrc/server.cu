// server.cu -- served SGBM (lumen_server_*): a request loop with continuous
// batching.  LumenStereo has no serving entry point (its callers loop over
// StereoSGBM::compute, tools/evaluate.cpp:158-160); this is the served form
// of that call.
//
//  * submit() validates a request, rejects one that can never fit the
//    device-memory budget (LUMEN_ERR_OUT_OF_BUDGET), copies its images into
//    pooled pinned host memory and queues it.  Rejections leave the server
//    serving.
//  * One server thread admits queued requests in arrival order as their
//    bytes (images, cost volume, sums, selections, rings: the same buffers as
//    the plain call) fit into a device arena of `budget` bytes allocated once,
//    up to `max_batch_pairs` per batch, whenever one of `max_inflight` batch
//    slots is free.  A batch is uploaded, rectified through the resident maps
//    of its calibration id (lumen_rectifier), and computed by the batched
//    launch core (batch_core.cuh): per pair cost volumes on the slot's
//    stream, one persistent sweep launch per kernel class, per pair
//    selection, and the copy back.  Schedule 4's sweep launches go to the
//    server's aggregation stream (sweep launches of different batches never
//    overlap, so each one's resident CTAs cover its hand-off window);
//    schedule 6's bands wait only on earlier bands of their own launch, so
//    its sweeps stay on the slot's stream and batches overlap entirely.  A
//    batch admitted while another is on the GPU overlaps with it: its
//    uploads and cost volumes run beside the other's sweep.
//  * The thread retires batches whose completion event has fired: results go
//    to the callers' buffers, arena slices are freed, waiters are woken.  A
//    batch still running after `watchdog_ms` has its requests completed with
//    LUMEN_ERR_TIMEOUT; its device memory stays reserved until the GPU work
//    really ends.
// Every request's output equals lumen_sgbm_compute's for the same (rectified)
// pair bit for bit, whatever it was batched with.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/lumen_sgbm.h"
#include "batch_core.cuh"
#include "host_arena.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace lumen;
using Clock = std::chrono::steady_clock;

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Pinned host buffers recycled by exact size (the sizes of a stream repeat).
class PinnedPool {
  public:
    ~PinnedPool() {
        for (auto& kv : free_)
            for (void* p : kv.second) cudaFreeHost(p);
    }
    void* get(size_t n) {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto it = free_.find(n);
            if (it != free_.end() && !it->second.empty()) {
                void* p = it->second.back();
                it->second.pop_back();
                return p;
            }
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, n, cudaHostAllocPortable) != cudaSuccess) return nullptr;
        return p;
    }
    void put(void* p, size_t n) {
        if (!p) return;
        std::lock_guard<std::mutex> g(mu_);
        free_[n].push_back(p);
    }

  private:
    std::mutex mu_;
    std::map<size_t, std::vector<void*>> free_;
};

struct Request {
    unsigned long long id = 0;
    lumen_stereo_params p{};
    int calib = -1;
    int W = 0, H = 0;
    uint8_t* in = nullptr;  // pinned: left then right, W*H bytes each
    int16_t* out = nullptr;  // pinned: the disparity map
    int16_t* user = nullptr;
    size_t need = 0, off = 0;
    Clock::time_point tSubmit, tAdmit, tDone;
    lumen_status status = LUMEN_OK;
    std::string err;
    double deviceMs = 0;
    int batchPairs = 0;
    unsigned long long batchId = 0;
    bool done = false;
    bool inFlight = false;  // its device work may still run (watchdog)
};

struct Slot {
    cudaStream_t s = nullptr;
    cudaEvent_t evStart = nullptr, evDone = nullptr;
    std::vector<cudaEvent_t> evs;  // sweep ordering, 2 per group
    int* dStatus = nullptr;
    int* hStatus = nullptr;  // pinned
    uint8_t* dDesc = nullptr;
    size_t descCap = 0;
    uint8_t* hDesc = nullptr;  // pinned
    size_t hDescCap = 0;
    std::vector<Request*> reqs;
    std::vector<BatchPair> pairs;
    std::vector<BatchGroup> groups;
    bool busy = false;
    bool expired = false;  // the watchdog completed its requests
    Clock::time_point tLaunch;
    unsigned long long batchId = 0;
};

size_t image_bytes(int W, int H) { return align256((size_t)W * H); }

}  // namespace

struct lumen_server {
    lumen_server_options opt{};
    int device = 0;
    int numSMs = 148;
    uint8_t* arenaBase = nullptr;
    Arena arena;
    PinnedPool pinned;
    uint32_t* magic = nullptr;
    cudaStream_t agg = nullptr;
    std::vector<Slot> slots;
    struct Calib {
        lumen_rectifier* rect;  // maps uploaded from the host, or
        float* maps;            // [4][H][W] maps generated on the device
        int W, H;
    };
    std::map<int, Calib> calib;
    std::mutex calibMu;

    std::mutex mu;  // queue, requests, stats
    std::condition_variable cvWork, cvDone;
    std::deque<Request*> queue;
    std::unordered_map<unsigned long long, Request*> reqs;
    unsigned long long nextId = 1, nextBatch = 1;
    bool stop = false;
    lumen_server_stats st{};
    std::thread thread;
    std::string fatal;  // a CUDA error that stopped the loop
    lumen_sgbm* plain = nullptr;  // the plain call of the fallback (server thread only)
    int failNext = 0;             // injected batch-launch failures still to come (S->mu)
};

namespace {

lumen_status sfail(lumen_status s, const std::string& m) { return set_error(s, m); }

// Bytes of a request's slice: images (raw copies too when rectified), the
// output map, then the working buffers of the batched launch core.
size_t request_bytes(const BatchPair& q, int calib, int sched, int R) {
    const size_t img = image_bytes(q.W, q.H);
    return 2 * img + (calib >= 0 ? 2 * img : 0) + align256((size_t)q.W * q.H * 2) + batch_pair_bytes(q, sched, R);
}

void complete(lumen_server* S, Request* r, lumen_status st, const std::string& err) {
    r->status = st;
    r->err = err;
    r->tDone = Clock::now();
    r->done = true;
    if (st == LUMEN_OK) S->st.completed++;
    else S->st.failed++;
}

// The request's images and output inside its arena slice, its raw input
// uploaded and rectified on stream `s` when it has a calibration: the first
// steps of a batch launch, and of the plain-call fallback.
struct ReqBufs {
    uint8_t* dl;
    uint8_t* dr;
    int16_t* dOut;
    size_t used;  // bytes of the slice these take (the batch core's buffers follow)
};

lumen_status stage_request(lumen_server* S, Request* r, cudaStream_t s, ReqBufs* out) {
    uint8_t* base = S->arenaBase + r->off;
    const size_t img = image_bytes(r->W, r->H), n = (size_t)r->W * r->H;
    uint8_t* dl = base;
    uint8_t* dr = base + img;
    size_t o = 2 * img;
    uint8_t* raw = nullptr;
    if (r->calib >= 0) {
        raw = base + o;
        o += 2 * img;
    }
    int16_t* dOut = reinterpret_cast<int16_t*>(base + o);
    o += align256(n * 2);
    uint8_t* up = raw ? raw : dl;
    if (cudaMemcpyAsync(up, r->in, n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(up + img, r->in + n, n, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return sfail(LUMEN_ERR_CUDA, "server: input upload failed");
    if (raw) {
        lumen_server::Calib c{};
        {
            std::lock_guard<std::mutex> g(S->calibMu);
            c = S->calib[r->calib];
        }
        if (c.maps) {
            const size_t m = (size_t)r->W * r->H;
            launch_remap(raw, raw + img, c.maps, c.maps + m, c.maps + 2 * m, c.maps + 3 * m, dl, dr, r->W, r->H, 1,
                         2, s);
            if (cudaGetLastError() != cudaSuccess) return sfail(LUMEN_ERR_CUDA, "server: remap launch failed");
        } else {
            lumen_status rs = lumen_rectifier_rectify_device(c.rect, raw, raw + img, 1, dl, dr, s);
            if (rs != LUMEN_OK) return rs;
        }
    }
    *out = ReqBufs{dl, dr, dOut, o};
    return LUMEN_OK;
}

// The plain-call fallback for one request of a failed batch (server thread,
// the request's arena slice still reserved, nothing of the batch still
// running on the device): staged again from the pinned input, computed by
// lumen_sgbm_compute_device with the default wait limit, copied to the
// caller's buffer.  Blocks the server loop while it runs.
lumen_status plain_fallback(lumen_server* S, Request* r, cudaStream_t s) {
    lumen_status st = LUMEN_OK;
    if (!S->plain) st = lumen_sgbm_create(&r->p, &S->plain);
    else st = lumen_sgbm_set_params(S->plain, &r->p);
    if (st != LUMEN_OK) return st;
    ReqBufs q{};
    st = stage_request(S, r, s, &q);
    if (st != LUMEN_OK) return st;
    st = lumen_sgbm_compute_device(S->plain, q.dl, q.dr, r->W, r->H, (size_t)r->W, 1, q.dOut,
                                   (size_t)r->W * 2, s);
    if (st != LUMEN_OK) return st;
    const size_t n = (size_t)r->W * r->H;
    if (cudaMemcpyAsync(r->out, q.dOut, n * 2, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return sfail(LUMEN_ERR_CUDA, "server: plain-call fallback failed");
    std::memcpy(r->user, r->out, n * 2);
    return LUMEN_OK;
}

lumen_status slot_launch(lumen_server* S, Slot& sl, std::vector<Request*>& adm) {
    const int R = S->opt.rows_per_band;
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (S->failNext > 0) {
            --S->failNext;
            return sfail(LUMEN_ERR_CUDA, "server: batch launch failed (injected)");
        }
    }
    sl.tLaunch = Clock::now();  // the watchdog counts from the start of the enqueue
    sl.reqs = adm;
    sl.pairs.clear();
    sl.groups.clear();
    sl.batchId = S->nextBatch++;
    for (Request* r : adm) {
        ReqBufs b{};
        lumen_status rs = stage_request(S, r, sl.s, &b);
        if (rs != LUMEN_OK) return rs;
        BatchPair q;
        lumen_status ps = batch_pair_init(q, &r->p, b.dl, b.dr, r->W, r->H, b.dOut);
        if (ps != LUMEN_OK) return ps;
        q.base = S->arenaBase + r->off;
        size_t o = b.used;
        batch_pair_layout(q, S->opt.schedule, R, o);
        sl.pairs.push_back(q);
    }
    std::vector<int> idx(sl.pairs.size());
    for (int i = 0; i < (int)idx.size(); ++i) idx[i] = i;
    batch_group_by_class(sl.pairs, idx, sl.groups);
    std::vector<uint8_t> host;
    lumen_status ds = batch_describe(sl.pairs, sl.groups, S->opt.schedule, R, S->numSMs, host);
    if (ds != LUMEN_OK) return ds;
    if (host.size() > sl.descCap) {
        if (sl.dDesc) cudaFree(sl.dDesc);
        sl.descCap = std::max<size_t>(host.size(), 1 << 20);
        if (cudaMalloc(&sl.dDesc, sl.descCap) != cudaSuccess) {
            sl.dDesc = nullptr;
            sl.descCap = 0;
            return sfail(LUMEN_ERR_CUDA, "server: descriptor allocation failed");
        }
    }
    if (host.size() > sl.hDescCap) {
        if (sl.hDesc) cudaFreeHost(sl.hDesc);
        sl.hDescCap = std::max<size_t>(host.size(), 1 << 20);
        if (cudaHostAlloc(&sl.hDesc, sl.hDescCap, cudaHostAllocPortable) != cudaSuccess) {
            sl.hDesc = nullptr;
            sl.hDescCap = 0;
            return sfail(LUMEN_ERR_CUDA, "server: pinned descriptor allocation failed");
        }
    }
    std::memcpy(sl.hDesc, host.data(), host.size());
    if (cudaMemcpyAsync(sl.dDesc, sl.hDesc, host.size(), cudaMemcpyHostToDevice, sl.s) != cudaSuccess)
        return sfail(LUMEN_ERR_CUDA, "server: descriptor upload failed");
    while (sl.evs.size() < 2 * sl.groups.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return sfail(LUMEN_ERR_CUDA, "server: event creation failed");
        sl.evs.push_back(e);
    }
    cudaEventRecord(sl.evStart, sl.s);
    unsigned long long nl = 0;
    lumen_status es = batch_enqueue_groups(sl.pairs, sl.groups, sl.dDesc, S->magic, sl.dStatus,
                                           S->opt.spin_limit ? S->opt.spin_limit : (1ll << 24), sl.s,
                                           S->opt.schedule == 6 ? nullptr : S->agg, sl.evs.data(), &nl);
    if (es != LUMEN_OK) return es;
    for (size_t i = 0; i < adm.size(); ++i) {
        const size_t n = (size_t)adm[i]->W * adm[i]->H;
        if (cudaMemcpyAsync(adm[i]->out, sl.pairs[i].out, n * 2, cudaMemcpyDeviceToHost, sl.s) != cudaSuccess)
            return sfail(LUMEN_ERR_CUDA, "server: result download failed");
    }
    cudaMemcpyAsync(sl.hStatus, sl.dStatus, sizeof(int), cudaMemcpyDeviceToHost, sl.s);
    cudaMemsetAsync(sl.dStatus, 0, sizeof(int), sl.s);
    if (cudaEventRecord(sl.evDone, sl.s) != cudaSuccess) return sfail(LUMEN_ERR_CUDA, "server: event record failed");
    sl.busy = true;
    sl.expired = false;
    return LUMEN_OK;
}

// Returns the requests' memory and finishes the ones the watchdog has not;
// when the batch's device-side waits ran out, those go through the plain-call
// fallback first (if enabled).
void slot_retire(lumen_server* S, Slot& sl) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, sl.evStart, sl.evDone);
    const int dev = *sl.hStatus;
    std::vector<lumen_status> fb(sl.reqs.size(), LUMEN_OK);
    if (dev != 0 && S->opt.plain_fallback) {
        // only the server thread completes requests, so `done` is stable here
        for (size_t i = 0; i < sl.reqs.size(); ++i)
            if (!sl.reqs[i]->done) fb[i] = plain_fallback(S, sl.reqs[i], sl.s);
    }
    std::lock_guard<std::mutex> g(S->mu);
    size_t idx = 0;
    for (Request* r : sl.reqs) {
        const lumen_status f = fb[idx++];
        r->inFlight = false;
        S->arena.release(r->off, r->need);
        S->st.admitted_bytes -= r->need;
        if (!r->done) {
            r->deviceMs = ms;
            if (dev == 0) {
                std::memcpy(r->user, r->out, (size_t)r->W * r->H * 2);
                complete(S, r, LUMEN_OK, "");
            } else if (S->opt.plain_fallback) {
                if (f == LUMEN_OK) S->st.fallbacks++;
                complete(S, r, f, f == LUMEN_OK ? "" : "the plain-call fallback of a timed-out batch failed");
            } else {
                complete(S, r, static_cast<lumen_status>(dev), "a bounded device-side wait timed out in a served batch");
            }
        }
        S->pinned.put(r->in, (size_t)r->W * r->H * 2);
        S->pinned.put(r->out, (size_t)r->W * r->H * 2);
        r->in = nullptr;
        r->out = nullptr;
        if (r->done && r->user == nullptr) {  // abandoned by its caller
            S->reqs.erase(r->id);
            delete r;
        }
    }
    sl.reqs.clear();
    sl.busy = false;
    S->st.inflight_batches--;
    S->cvDone.notify_all();
    S->cvWork.notify_all();
}

// A fatal CUDA error: every request still in a busy slot completes with
// LUMEN_ERR_CUDA and leaves its slot; the device memory is not reused (the
// server stops).  Caller holds S->mu.
void fail_all_inflight(lumen_server* S) {
    for (Slot& o : S->slots) {
        if (!o.busy) continue;
        for (Request* r : o.reqs) {
            r->inFlight = false;
            if (!r->done) {
                complete(S, r, LUMEN_ERR_CUDA, S->fatal);
            } else if (r->user == nullptr) {  // abandoned by its caller after the watchdog
                S->reqs.erase(r->id);
                delete r;
            }
        }
        o.reqs.clear();
        o.busy = false;
        S->st.inflight_batches--;
    }
}

void server_loop(lumen_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        bool progressed = false;
        for (Slot& sl : S->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.evDone);
            if (q == cudaSuccess) {
                slot_retire(S, sl);
                progressed = true;
            } else if (q != cudaErrorNotReady) {
                // the context is unusable: fail every request of every busy
                // slot and of the queue, and stop serving
                std::lock_guard<std::mutex> g(S->mu);
                S->fatal = std::string("server: CUDA error: ") + cudaGetErrorString(q);
                fail_all_inflight(S);
                for (Request* r : S->queue) complete(S, r, LUMEN_ERR_CUDA, S->fatal);
                S->queue.clear();
                S->stop = true;
                S->cvDone.notify_all();
                return;
            } else if (S->opt.watchdog_ms > 0 && !sl.expired &&
                       ms_between(sl.tLaunch, Clock::now()) > S->opt.watchdog_ms) {
                std::lock_guard<std::mutex> g(S->mu);
                for (Request* r : sl.reqs)
                    if (!r->done) complete(S, r, LUMEN_ERR_TIMEOUT, "server: the batch missed the watchdog deadline");
                sl.expired = true;
                S->st.watchdog_expired++;
                S->cvDone.notify_all();
            }
        }
        Slot* freeSlot = nullptr;
        for (Slot& sl : S->slots)
            if (!sl.busy) { freeSlot = &sl; break; }
        std::vector<Request*> adm;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            bool anyBusy = false;
            for (Slot& sl : S->slots) anyBusy |= sl.busy;
            if (S->stop && S->queue.empty() && !anyBusy) return;
            if (freeSlot) {
                while (!S->queue.empty() && (int)adm.size() < S->opt.max_batch_pairs) {
                    Request* r = S->queue.front();
                    size_t off = 0;
                    if (!S->arena.alloc(r->need, &off)) break;  // wait for memory, in arrival order
                    r->off = off;
                    r->tAdmit = Clock::now();
                    r->inFlight = true;
                    S->queue.pop_front();
                    S->st.admitted_bytes += r->need;
                    S->st.peak_admitted_bytes = std::max(S->st.peak_admitted_bytes, S->st.admitted_bytes);
                    adm.push_back(r);
                }
                S->st.queue_depth = (int)S->queue.size();
                if (!adm.empty()) {
                    S->st.batches++;
                    S->st.inflight_batches++;
                    S->st.peak_batch_pairs = std::max<int>(S->st.peak_batch_pairs, (int)adm.size());
                }
            }
            if (adm.empty() && !progressed) {
                // nothing to start or retire: sleep until a submit, or poll
                // the running batches again shortly
                S->cvWork.wait_for(lk, anyBusy ? std::chrono::microseconds(50) : std::chrono::milliseconds(5));
                continue;
            }
        }
        if (!adm.empty()) {
            const unsigned long long bid = S->nextBatch;
            lumen_status ls = slot_launch(S, *freeSlot, adm);
            std::unique_lock<std::mutex> g(S->mu);
            for (Request* r : adm) {
                r->batchPairs = (int)adm.size();
                r->batchId = bid;
            }
            if (ls != LUMEN_OK) {
                // nothing of this batch may still be queued on the device once
                // its memory is reused (or the fallback reuses it)
                cudaStreamSynchronize(freeSlot->s);
                cudaStreamSynchronize(S->agg);
                std::vector<lumen_status> fb(adm.size(), ls);
                if (S->opt.plain_fallback) {
                    g.unlock();   // the fallback runs device work: submitters keep going meanwhile
                    for (size_t i = 0; i < adm.size(); ++i) fb[i] = plain_fallback(S, adm[i], freeSlot->s);
                    g.lock();
                }
                for (size_t i = 0; i < adm.size(); ++i) {
                    Request* r = adm[i];
                    S->arena.release(r->off, r->need);
                    S->st.admitted_bytes -= r->need;
                    r->inFlight = false;
                    if (fb[i] == LUMEN_OK) S->st.fallbacks++;
                    complete(S, r, fb[i], fb[i] == LUMEN_OK ? "" : "server: batch launch failed");
                }
                freeSlot->busy = false;
                S->st.inflight_batches--;
                S->cvDone.notify_all();
            }
        }
    }
}

}  // namespace

extern "C" void lumen_server_options_default(lumen_server_options* o) {
    if (!o) return;
    *o = lumen_server_options{};
    o->device_budget_bytes = 40ull << 30;
    o->max_batch_pairs = 32;
    o->rows_per_band = 16;
    o->max_inflight = 2;
    o->watchdog_ms = 60000;
    o->spin_limit = 0;
    o->plain_fallback = 1;
    o->schedule = 6;
}

extern "C" lumen_status lumen_server_create(const lumen_server_options* opt, lumen_server** out) {
    if (!out) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_server_create: out is NULL");
    *out = nullptr;
    lumen_server_options o;
    lumen_server_options_default(&o);
    if (opt) o = *opt;
    if (o.device_budget_bytes < (1u << 20)) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "budget below 1 MiB");
    if (o.max_batch_pairs < 1 || o.max_batch_pairs > 4095)
        return sfail(LUMEN_ERR_INVALID_ARGUMENT, "max_batch_pairs must be in [1, 4095]");
    if (o.schedule != 4 && o.schedule != 6) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "schedule must be 4 or 6");
    if (!batch_rows_valid(o.schedule, o.rows_per_band))
        return sfail(LUMEN_ERR_INVALID_ARGUMENT,
                     "rows_per_band must be 4, 8 or 16 with schedule 4, 16, 24 or 32 with schedule 6");
    if (o.max_inflight < 1 || o.max_inflight > 8) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "max_inflight must be in [1, 8]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return sfail(LUMEN_ERR_NO_DEVICE, "no CUDA device available");
    std::unique_ptr<lumen_server> S(new lumen_server());
    S->opt = o;
    cudaGetDevice(&S->device);
    cudaDeviceGetAttribute(&S->numSMs, cudaDevAttrMultiProcessorCount, S->device);
    auto bad = [&](cudaError_t e, const char* what) {
        return sfail(LUMEN_ERR_CUDA, std::string("lumen_server_create: ") + what + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaMalloc(&S->arenaBase, o.device_budget_bytes);
    if (e != cudaSuccess) {
        S->arenaBase = nullptr;
        lumen_server_destroy(S.release());
        return bad(e, "device arena");
    }
    S->arena.reset(o.device_budget_bytes);
    S->st.budget_bytes = o.device_budget_bytes;
    e = cudaMalloc(&S->magic, 443 * sizeof(uint32_t));
    if (e == cudaSuccess) e = launch_magic(S->magic, 443, 0);
    int prLeast = 0, prGreatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
    // sweeps first: their CTAs wait on one another, the other kernels do not
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&S->agg, cudaStreamNonBlocking, prGreatest);
    S->slots.resize(o.max_inflight);
    for (Slot& sl : S->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.evStart);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.evDone);
        if (e == cudaSuccess) e = cudaMalloc(&sl.dStatus, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(sl.dStatus, 0, sizeof(int));
        if (e == cudaSuccess) e = cudaHostAlloc(&sl.hStatus, sizeof(int), cudaHostAllocPortable);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        lumen_server_destroy(S.release());
        return bad(e, "setup");
    }
    lumen_server* raw = S.release();
    raw->thread = std::thread(server_loop, raw);
    *out = raw;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_destroy(lumen_server* S) {
    if (!S) return LUMEN_OK;
    if (S->thread.joinable()) {
        {
            std::lock_guard<std::mutex> g(S->mu);
            S->stop = true;
        }
        S->cvWork.notify_all();
        S->thread.join();
    }
    cudaDeviceSynchronize();
    for (auto& kv : S->reqs) {
        Request* r = kv.second;
        S->pinned.put(r->in, (size_t)r->W * r->H * 2);
        S->pinned.put(r->out, (size_t)r->W * r->H * 2);
        delete r;
    }
    for (Slot& sl : S->slots) {
        if (sl.s) cudaStreamDestroy(sl.s);
        if (sl.evStart) cudaEventDestroy(sl.evStart);
        if (sl.evDone) cudaEventDestroy(sl.evDone);
        for (cudaEvent_t ev : sl.evs) cudaEventDestroy(ev);
        if (sl.dStatus) cudaFree(sl.dStatus);
        if (sl.hStatus) cudaFreeHost(sl.hStatus);
        if (sl.dDesc) cudaFree(sl.dDesc);
        if (sl.hDesc) cudaFreeHost(sl.hDesc);
    }
    for (auto& kv : S->calib) {
        if (kv.second.rect) lumen_rectifier_destroy(kv.second.rect);
        if (kv.second.maps) cudaFree(kv.second.maps);
    }
    if (S->plain) lumen_sgbm_destroy(S->plain);
    if (S->agg) cudaStreamDestroy(S->agg);
    if (S->magic) cudaFree(S->magic);
    if (S->arenaBase) cudaFree(S->arenaBase);
    delete S;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_set_calibration(lumen_server* S, int calib_id, int width, int height,
                                                     const float* map0x, const float* map0y,
                                                     const float* map1x, const float* map1y) {
    if (!S) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL server");
    if (calib_id < 0) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "calibration ids are >= 0");
    lumen_rectifier* r = nullptr;
    lumen_status st = lumen_rectifier_create(width, height, map0x, map0y, map1x, map1y, &r);
    if (st != LUMEN_OK) return st;
    std::lock_guard<std::mutex> g(S->calibMu);
    if (S->calib.count(calib_id)) {
        // queued or running requests may use the registered maps: an id is
        // bound once for the server's lifetime
        lumen_rectifier_destroy(r);
        return sfail(LUMEN_ERR_INVALID_ARGUMENT, "calibration id already registered");
    }
    S->calib[calib_id] = lumen_server::Calib{r, nullptr, width, height};
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_set_calibration_params(lumen_server* S, int calib_id, int width, int height,
                                                            const double K0[9], const double D0[5],
                                                            const double R0[9], const double P0[12],
                                                            const double K1[9], const double D1[5],
                                                            const double R1[9], const double P1[12]) {
    if (!S) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL server");
    if (calib_id < 0) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "calibration ids are >= 0");
    if (width <= 0 || height <= 0) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "empty calibration image size");
    {
        std::lock_guard<std::mutex> g(S->calibMu);
        if (S->calib.count(calib_id)) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "calibration id already registered");
    }
    const size_t m = (size_t)width * height;
    float* maps = nullptr;
    cudaError_t e = cudaMalloc(&maps, 4 * m * sizeof(float));
    if (e != cudaSuccess) return sfail(LUMEN_ERR_CUDA, std::string("calibration maps: ") + cudaGetErrorString(e));
    cudaStream_t s = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    lumen_status st = e == cudaSuccess ? LUMEN_OK : sfail(LUMEN_ERR_CUDA, "calibration stream");
    if (st == LUMEN_OK) st = lumen_rectify_maps_device(K0, D0, R0, P0, width, height, maps, maps + m, s);
    if (st == LUMEN_OK) st = lumen_rectify_maps_device(K1, D1, R1, P1, width, height, maps + 2 * m, maps + 3 * m, s);
    if (st == LUMEN_OK && cudaStreamSynchronize(s) != cudaSuccess) st = sfail(LUMEN_ERR_CUDA, "calibration maps");
    if (s) cudaStreamDestroy(s);
    if (st != LUMEN_OK) {
        cudaFree(maps);
        return st;
    }
    std::lock_guard<std::mutex> g(S->calibMu);
    if (S->calib.count(calib_id)) {
        cudaFree(maps);
        return sfail(LUMEN_ERR_INVALID_ARGUMENT, "calibration id already registered");
    }
    S->calib[calib_id] = lumen_server::Calib{nullptr, maps, width, height};
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_submit(lumen_server* S, const lumen_stereo_params* p, int calib_id,
                                            const uint8_t* left, const uint8_t* right, int width, int height,
                                            int16_t* out, unsigned long long* request_id) {
    if (!S || !p || !request_id) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_server_submit: NULL argument");
    *request_id = 0;
    if (!left || !right || !out) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "Input images are empty");
    BatchPair q;
    // validation only: the device pointers are bound at admission
    static const uint8_t probe[1] = {0};
    lumen_status st = batch_pair_init(q, p, probe, probe, width, height, reinterpret_cast<int16_t*>(1));
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->st.submitted++;
        if (st != LUMEN_OK) S->st.rejected++;
    }
    if (st != LUMEN_OK) return st;
    if (calib_id >= 0) {
        std::lock_guard<std::mutex> g(S->calibMu);
        auto it = S->calib.find(calib_id);
        if (it == S->calib.end() || it->second.W != width || it->second.H != height) {
            std::lock_guard<std::mutex> g2(S->mu);
            S->st.rejected++;
            return sfail(LUMEN_ERR_INVALID_ARGUMENT,
                         it == S->calib.end() ? "unknown calibration id"
                                              : "image size differs from the calibration's");
        }
    }
    Request* r = new Request();
    r->p = *p;
    r->calib = calib_id;
    r->W = width;
    r->H = height;
    r->need = request_bytes(q, calib_id, S->opt.schedule, S->opt.rows_per_band);
    if (r->need > S->opt.device_budget_bytes) {
        delete r;
        std::lock_guard<std::mutex> g(S->mu);
        S->st.rejected++;
        return sfail(LUMEN_ERR_OUT_OF_BUDGET, "request needs more device memory than the server's budget");
    }
    const size_t n = (size_t)width * height;
    r->in = static_cast<uint8_t*>(S->pinned.get(2 * n));
    r->out = static_cast<int16_t*>(S->pinned.get(2 * n));
    if (!r->in || !r->out) {
        S->pinned.put(r->in, 2 * n);
        S->pinned.put(r->out, 2 * n);
        delete r;
        return sfail(LUMEN_ERR_CUDA, "pinned host allocation failed");
    }
    std::memcpy(r->in, left, n);
    std::memcpy(r->in + n, right, n);
    r->user = out;
    r->tSubmit = Clock::now();
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (S->stop) {
            S->pinned.put(r->in, 2 * n);
            S->pinned.put(r->out, 2 * n);
            delete r;
            return sfail(LUMEN_ERR_CUDA, S->fatal.empty() ? "server is stopping" : S->fatal);
        }
        r->id = S->nextId++;
        S->reqs[r->id] = r;
        S->queue.push_back(r);
        S->st.queue_depth = (int)S->queue.size();
        S->st.peak_queue_depth = std::max(S->st.peak_queue_depth, S->st.queue_depth);
        *request_id = r->id;
    }
    S->cvWork.notify_all();
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_wait(lumen_server* S, unsigned long long id, int timeout_ms,
                                          lumen_request_info* info) {
    if (!S) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "unknown request id");
    Request* r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) S->cvDone.wait(lk, ready);
    else if (!S->cvDone.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return sfail(LUMEN_ERR_TIMEOUT, "request not finished within the wait's timeout");
    if (info) {
        info->status = r->status;
        info->latency_ms = ms_between(r->tSubmit, r->tDone);
        info->queue_ms = r->tAdmit.time_since_epoch().count() ? ms_between(r->tSubmit, r->tAdmit) : 0.0;
        info->device_ms = r->deviceMs;
        info->batch_pairs = r->batchPairs;
        info->batch_id = r->batchId;
    }
    const lumen_status st = r->status;
    const std::string err = r->err;
    if (r->inFlight) {
        r->user = nullptr;  // the retire step frees it
    } else {
        S->reqs.erase(it);
        delete r;
    }
    lk.unlock();
    if (st != LUMEN_OK) return sfail(st, err);
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_debug_fail_batches(lumen_server* S, int n) {
    if (!S || n < 0) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "lumen_server_debug_fail_batches: bad argument");
    std::lock_guard<std::mutex> g(S->mu);
    S->failNext = n;
    return LUMEN_OK;
}

extern "C" lumen_status lumen_server_get_stats(lumen_server* S, lumen_server_stats* out) {
    if (!S || !out) return sfail(LUMEN_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> g(S->mu);
    *out = S->st;
    return LUMEN_OK;
}
