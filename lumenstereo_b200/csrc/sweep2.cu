// sweep2.cu -- host side of schedule 3 (decoupled-row fused sweeps,
// sweep2_kernel.cuh): shared-memory fit, exchange sizing, launch.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "sweep2_kernel.cuh"

namespace lumen {

#define LUMEN_SWEEP2_DECL(KW)                                                                  \
    cudaError_t sweep2_dispatch_##KW(const Sweep2Args& a, int R, int NP, bool wrap, int smem,  \
                                     int grid, cudaStream_t s, int* perSM);
LUMEN_SWEEP2_DECL(1)
LUMEN_SWEEP2_DECL(2)
LUMEN_SWEEP2_DECL(3)
LUMEN_SWEEP2_DECL(4)
LUMEN_SWEEP2_DECL(5)
LUMEN_SWEEP2_DECL(6)
LUMEN_SWEEP2_DECL(7)
LUMEN_SWEEP2_DECL(8)

static cudaError_t dispatch2(const Sweep2Args& a, int R, int NP, bool wrap, int smem, int grid,
                             cudaStream_t s, int* perSM) {
    switch (a.Dp / 64) {
    case 1: return sweep2_dispatch_1(a, R, NP, wrap, smem, grid, s, perSM);
    case 2: return sweep2_dispatch_2(a, R, NP, wrap, smem, grid, s, perSM);
    case 3: return sweep2_dispatch_3(a, R, NP, wrap, smem, grid, s, perSM);
    case 4: return sweep2_dispatch_4(a, R, NP, wrap, smem, grid, s, perSM);
    case 5: return sweep2_dispatch_5(a, R, NP, wrap, smem, grid, s, perSM);
    case 6: return sweep2_dispatch_6(a, R, NP, wrap, smem, grid, s, perSM);
    case 7: return sweep2_dispatch_7(a, R, NP, wrap, smem, grid, s, perSM);
    case 8: return sweep2_dispatch_8(a, R, NP, wrap, smem, grid, s, perSM);
    default: return cudaErrorInvalidValue;
    }
}

int sweep2_rows_options(int Dp, int* out, int max) {
    (void)Dp;
    const int opts[] = {8, 4};
    int n = 0;
    for (int o : opts)
        if (n < max) out[n++] = o;
    return n;
}

static Sweep2Args base_args(const SgmConsts& k, int nBands, int M, int QB) {
    Sweep2Args a{};
    a.W = k.W; a.H = k.H; a.D = k.D; a.Dp = k.Dp;
    a.P1 = k.P1; a.P2 = k.P2; a.costScale = k.costScale;
    a.p1x2 = k.p1x2; a.bsub = k.bsub;
    a.nBands = nBands; a.M = M; a.QB = QB;
    return a;
}

cudaError_t sweep2_plan(const SgmConsts& k, int R, bool wrap, bool diag, int numSMs, Sweep2Plan* plan) {
    if (R != 4 && R != 8) return cudaErrorInvalidValue;
    const int NP = diag ? 3 : 1;
    int dev = 0, maxSmem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int QB = 16;
    Sweep2Smem L = sweep2_smem(k.W, k.Dp, R, NP, QB);
    if (L.total > maxSmem) {
        QB = 8;
        L = sweep2_smem(k.W, k.Dp, R, NP, QB);
    }
    if (L.total > maxSmem) return cudaErrorInvalidConfiguration;
    const int nBands = (k.H + R - 1) / R;
    Sweep2Args a = base_args(k, nBands, 2, QB);
    int perSM = 0;
    cudaError_t e = dispatch2(a, R, NP, wrap, L.total, 0, nullptr, &perSM);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorInvalidConfiguration;
    const int grid = std::min(2 * nBands, perSM * numSMs);
    // exchange rows: band b waits for band b-M+1 to have imported row b-M.
    // A band trails its predecessor by about 2R + 8 pixels, so
    // M ~ W / (2R + 8) keeps that wait off the critical path.
    int M = std::max(2, k.W / (2 * R + 8) + 4);
    const size_t SB = (size_t)sweep2_slot_bytes(k.Dp, NP);
    const size_t rowBytes = (size_t)k.W * SB;
    const size_t cap = (size_t)1 << 30;  // keep the exchange rows of both sweeps under 1 GiB
    while (M > 2 && 2 * (size_t)M * rowBytes > cap) --M;
    M = std::min(M, std::max(2, nBands));
    plan->R = R;
    plan->QB = QB;
    plan->nBands = nBands;
    plan->M = M;
    plan->grid = grid;
    plan->smem = L.total;
    plan->ringBytes = 2 * (size_t)M * rowBytes;
    plan->counterWords = 4 * (size_t)nBands + 32;
    return cudaSuccess;
}

cudaError_t launch_aggregate_sweep2(const PairView& pv, uint16_t* partB, const SgmConsts& k,
                                    bool wrap, bool diag, const Sweep2Plan& plan, uint8_t* xring,
                                    unsigned* counters, int* status, long long spinMax,
                                    cudaStream_t s, int stallTest) {
    Sweep2Args a = base_args(k, plan.nBands, plan.M, plan.QB);
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
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * plan.counterWords, s);
    if (e != cudaSuccess) return e;
    int dummy = 0;
    return dispatch2(a, plan.R, diag ? 3 : 1, wrap, plan.smem, plan.grid, s, &dummy);
}

}  // namespace lumen
