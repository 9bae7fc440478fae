// sweep.cu -- host side of the fused two-sweep aggregation (schedule 2):
// configuration choice, exchange-ring sizing and dispatch to the compiled
// instances in sweep_cfg_*.cu (kernel in sweep_kernel.cuh).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "sweep_kernel.cuh"

namespace lumen {

#define LUMEN_SWEEP_DISPATCH(dp)                                                           \
    cudaError_t sweep_dispatch_##dp(SweepArgs a, int T, int NW, bool wrap, bool diag,     \
                                    cudaStream_t s, int numSMs, int* g);
LUMEN_SWEEP_DISPATCH(64)
LUMEN_SWEEP_DISPATCH(128)
LUMEN_SWEEP_DISPATCH(192)
LUMEN_SWEEP_DISPATCH(256)
LUMEN_SWEEP_DISPATCH(320)
LUMEN_SWEEP_DISPATCH(384)
LUMEN_SWEEP_DISPATCH(448)
LUMEN_SWEEP_DISPATCH(512)

int sweep_configs(int Dp, SweepConfig* out, int max) {
    static const SweepConfig small[] = {{32, 4}, {32, 8}, {16, 4}, {8, 4}, {8, 2}};
    static const SweepConfig mid[] = {{32, 4}, {32, 8}, {16, 4}};
    static const SweepConfig big[] = {{32, 4}, {32, 8}};
    const SweepConfig* src = Dp <= 128 ? small : (Dp <= 256 ? mid : big);
    const int n = Dp <= 128 ? 5 : (Dp <= 256 ? 3 : 2);
    for (int i = 0; i < n && i < max; ++i) out[i] = src[i];
    return std::min(n, max);
}

SweepConfig sweep_default_config(int Dp, bool wrap) {
    (void)Dp;
    (void)wrap;
    return SweepConfig{32, 4};
}

static cudaError_t dispatch(const SweepArgs& a, SweepConfig c, bool wrap, bool diag, cudaStream_t s,
                            int numSMs, int* g) {
    switch (a.Dp) {
    case 64: return sweep_dispatch_64(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 128: return sweep_dispatch_128(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 192: return sweep_dispatch_192(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 256: return sweep_dispatch_256(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 320: return sweep_dispatch_320(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 384: return sweep_dispatch_384(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 448: return sweep_dispatch_448(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    case 512: return sweep_dispatch_512(a, c.T, c.NW, wrap, diag, s, numSMs, g);
    default: return cudaErrorInvalidValue;
    }
}

static SweepArgs make_args(const PairView& pv, uint16_t* partB, const SgmConsts& k, SweepConfig c) {
    SweepArgs a{};
    a.cost = pv.cost;
    a.img = pv.img;
    a.part[0] = pv.agg;
    a.part[1] = partB;
    a.W = k.W; a.H = k.H; a.D = k.D; a.Dp = k.Dp;
    a.P1 = k.P1; a.P2 = k.P2; a.costScale = k.costScale;
    a.p1x2 = k.p1x2; a.bsub = k.bsub;
    a.R = c.NW * 32 / c.T;
    a.nBands = (k.H + a.R - 1) / a.R;
    a.G = a.nBands;
    a.slotBytes = 2 * k.Dp + 16;
    return a;
}

bool sweep_fits(int W, int Dp, SweepConfig c) {
    int dev = 0, maxSmem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return sweep_smem(W, Dp, c.NW * 32 / c.T).total + 1024 <= maxSmem;
}

cudaError_t sweep_plan(const PairView& pv, const SgmConsts& k, SweepConfig c, bool wrap, bool diag,
                       int numSMs, SweepPlan* plan) {
    SweepArgs a = make_args(pv, nullptr, k, c);
    a.plan = 1;
    int G = 0;
    cudaError_t e = dispatch(a, c, wrap, diag, nullptr, numSMs, &G);
    if (e != cudaSuccess) return e;
    plan->G = G;
    plan->nBands = a.nBands;
    // one wave (every band resident): small rings with back-pressure; otherwise
    // a full row per ring so that a producer never waits inside its band
    plan->K = (G == a.nBands) ? std::min(k.W, 128) : k.W;
    plan->ringBytes = (size_t)2 * G * plan->K * 3 * (2 * k.Dp + 16);
    plan->counterWords = (size_t)4 * G;
    return cudaSuccess;
}

cudaError_t launch_aggregate_sweep(const PairView& pv, uint16_t* partB, const SgmConsts& k,
                                   bool wrap, bool diag, SweepConfig c, const SweepPlan& plan,
                                   uint8_t* xring, unsigned* counters, int* status,
                                   long long spinMax, cudaStream_t s, int numSMs) {
    SweepArgs a = make_args(pv, partB, k, c);
    a.xring = xring;
    a.prod = counters;
    a.cons = counters + 2 * plan.G;
    a.status = status;
    a.K = plan.K;
    a.spinMax = spinMax;
    a.plan = 0;
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * plan.counterWords, s);
    if (e != cudaSuccess) return e;
    int G = 0;
    e = dispatch(a, c, wrap, diag, s, numSMs, &G);
    if (e == cudaSuccess && G != plan.G) return cudaErrorInvalidConfiguration;
    return e;
}

}  // namespace lumen
