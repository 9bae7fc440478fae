// wave.cu -- host side of schedule 4 (lockstep row-band fused sweeps with lane teams,
// wave_kernel.cuh): shared-memory fit, exchange sizing, launch.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "wave_kernel.cuh"

namespace lumen {

#define LUMEN_WAVE_DECL(KW)                                                                    \
    cudaError_t wave_dispatch_##KW(const WaveArgs& a, int R, int NP, bool wrap, int smem,      \
                                   int grid, cudaStream_t s, int* perSM);
LUMEN_WAVE_DECL(1)
LUMEN_WAVE_DECL(2)
LUMEN_WAVE_DECL(3)
LUMEN_WAVE_DECL(4)
LUMEN_WAVE_DECL(5)
LUMEN_WAVE_DECL(6)
LUMEN_WAVE_DECL(7)
LUMEN_WAVE_DECL(8)

static cudaError_t dispatch_wave(const WaveArgs& a, int R, int NP, bool wrap, int smem, int grid,
                                 cudaStream_t s, int* perSM) {
    switch (a.Dp / 64) {
    case 1: return wave_dispatch_1(a, R, NP, wrap, smem, grid, s, perSM);
    case 2: return wave_dispatch_2(a, R, NP, wrap, smem, grid, s, perSM);
    case 3: return wave_dispatch_3(a, R, NP, wrap, smem, grid, s, perSM);
    case 4: return wave_dispatch_4(a, R, NP, wrap, smem, grid, s, perSM);
    case 5: return wave_dispatch_5(a, R, NP, wrap, smem, grid, s, perSM);
    case 6: return wave_dispatch_6(a, R, NP, wrap, smem, grid, s, perSM);
    case 7: return wave_dispatch_7(a, R, NP, wrap, smem, grid, s, perSM);
    case 8: return wave_dispatch_8(a, R, NP, wrap, smem, grid, s, perSM);
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

static WaveArgs wave_base_args(const SgmConsts& k, int nBands, int Q) {
    WaveArgs a{};
    a.W = k.W; a.H = k.H; a.D = k.D; a.Dp = k.Dp;
    a.P1 = k.P1; a.P2 = k.P2; a.costScale = k.costScale;
    a.p1x2 = k.p1x2; a.bsub = k.bsub;
    a.nBands = nBands;
    a.QI = Q;
    a.QX = Q;
    return a;
}

cudaError_t wave_plan(const SgmConsts& k, int R, bool wrap, bool diag, int numSMs, WavePlan* plan) {
    if (R != 4 && R != 8 && R != 16) return cudaErrorInvalidValue;
    const int NP = diag ? 3 : 1;
    int dev = 0, maxSmem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // largest helper rings that fit
    int Q = 0;
    WaveSmem L{};
    for (int q : {16, 8}) {
        L = wave_smem(k.W, k.Dp, R, NP, q, q);
        if (L.total <= maxSmem) {
            Q = q;
            break;
        }
    }
    if (!Q) return cudaErrorInvalidConfiguration;
    const int nBands = (k.H + R - 1) / R;
    WaveArgs a = wave_base_args(k, nBands, Q);
    int perSM = 0;
    cudaError_t e = dispatch_wave(a, R, NP, wrap, L.total, 0, nullptr, &perSM);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    plan->R = R;
    plan->Q = Q;
    plan->nBands = nBands;
    plan->grid = std::min(2 * nBands, perSM * numSMs);
    plan->smem = L.total;
    plan->ringBytes = 2 * (size_t)nBands * kWK * (size_t)wave_slot_bytes(k.Dp, NP);
    plan->counterWords = 4 * (size_t)nBands + 32;
    return cudaSuccess;
}

cudaError_t launch_aggregate_wave(const PairView& pv, uint16_t* partB, const SgmConsts& k,
                                  bool wrap, bool diag, const WavePlan& plan, uint8_t* xring,
                                  unsigned* counters, int* status, long long spinMax,
                                  cudaStream_t s, int stallTest, unsigned long long* trace) {
    WaveArgs a = wave_base_args(k, plan.nBands, plan.Q);
    a.cost = pv.cost;
    a.img = pv.img;
    a.part[0] = pv.agg;
    a.part[1] = partB;
    a.xring = xring;
    a.prod = counters;
    a.cons = counters + 2 * plan.nBands;
    a.ticket = counters + 4 * plan.nBands;
    a.status = status;
    a.spinMax = spinMax;
    a.stallTest = stallTest;
    a.trace = trace;
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * plan.counterWords, s);
    if (e != cudaSuccess) return e;
    int dummy = 0;
    return dispatch_wave(a, plan.R, diag ? 3 : 1, wrap, plan.smem, plan.grid, s, &dummy);
}

}  // namespace lumen
