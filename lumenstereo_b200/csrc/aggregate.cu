// aggregate.cu -- SGM aggregation, one kernel launch per path direction.
//
// Replaces aggregateCostHorizontalLR/RL, VerticalTB/BT (src/sgbm_kernels.cu:
// 315-514) and the four diagonal kernels (:519-742).  Every path line is
// walked by one warp with disparities across lanes (sgm_step.cuh), so a
// direction needs one launch instead of the reference's W+H-1 launches per
// diagonal direction, and no H*W*D L_diag scratch volume: the previous step's
// L lives in registers.  The first direction of a compute stores L into the
// aggregated volume, later ones add (mod 2^16); results do not depend on the
// direction order because uint16 addition is associative.
#include "common.cuh"
#include "kernels.cuh"
#include "sgm_step.cuh"

namespace lumen {

// First pixel and step of line `li` of direction `dir` (LR, RL, TB, BT, TLBR,
// BRTL, TRBL, BLTR).  Lines of one direction cover every pixel exactly once.
__device__ __forceinline__ void line_start(int dir, int li, int W, int H, int& x, int& y, int& sx,
                                           int& sy) {
    switch (dir) {
    case 0: x = 0; y = li; sx = 1; sy = 0; break;
    case 1: x = W - 1; y = li; sx = -1; sy = 0; break;
    case 2: x = li; y = 0; sx = 0; sy = 1; break;
    case 3: x = li; y = H - 1; sx = 0; sy = -1; break;
    case 4: if (li < W) { x = li; y = 0; } else { x = 0; y = li - W + 1; } sx = 1; sy = 1; break;
    case 5: if (li < W) { x = li; y = H - 1; } else { x = W - 1; y = li - W; } sx = -1; sy = -1; break;
    case 6: if (li < W) { x = li; y = 0; } else { x = W - 1; y = li - W + 1; } sx = -1; sy = 1; break;
    default: if (li < W) { x = li; y = H - 1; } else { x = 0; y = li - W; } sx = 1; sy = -1; break;
    }
}


// P2adj table (src/sgbm_kernels.cu:304-310): index |I[p] - I[p-r]| in [0,255].
__device__ __forceinline__ void fill_p2_lut(int* lut, int P1, int P2) {
    for (int g = threadIdx.x; g < 256; g += blockDim.x) lut[g] = max(P1 + 1, P2 * 8 / max(8, g));
}

// Number of pixels on the line that starts at (x, y) with step (sx, sy).
__device__ __forceinline__ int line_length(int x, int y, int sx, int sy, int W, int H) {
    int n = 1 << 30;
    if (sx > 0) n = min(n, W - x);
    if (sx < 0) n = min(n, x + 1);
    if (sy > 0) n = min(n, H - y);
    if (sy < 0) n = min(n, y + 1);
    return n;
}

// One warp per path line.  Loads of the cost and aggregated words (and the
// image byte) for pixel i+PF are issued while pixel i is computed: the
// recurrence's step chain never waits on DRAM latency.
template <int KW, bool WRAP, bool FULL, int PF>
__global__ void __launch_bounds__(128)
agg_dir_kernel(PairView pv, SgmConsts k, int dir, int first) {
    __shared__ int p2lut[256];
    fill_p2_lut(p2lut, k.P1, k.P2);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (li >= num_lines(dir, k.W, k.H)) return;
    int x0, y0, sx, sy;
    line_start(dir, li, k.W, k.H, x0, y0, sx, sy);
    const int len = line_length(x0, y0, sx, sy, k.W, k.H);
    LaneMasks<KW> mk;
    make_lane_masks<KW>(lane, k.D, mk);
    const size_t Dp = (size_t)k.Dp;
    const int off = lane * 2 * KW;
    const long long pstep = (long long)sy * k.W + sx;  // pixel index step along the line
    const long long p0 = (long long)y0 * k.W + x0;

    uint32_t cb[PF][KW], ab[PF][KW];
    int ib[PF];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
        if (j < len) {
            const size_t p = (size_t)(p0 + j * pstep);
            load_cost_words<KW>(pv.cost + p * Dp + off, cb[j]);
            if (!first) load_words<KW>(pv.agg + p * Dp + off, ab[j]);
            ib[j] = pv.img[p];
        }
    }
    uint32_t Lp[KW], Ln[KW], Cw[KW];
    uint32_t minPrev = 0;
    int prevI = 0;
    for (int base = 0; base < len; base += PF) {
#pragma unroll
        for (int j = 0; j < PF; ++j) {
            const int i = base + j;
            if (i >= len) break;
            const size_t p = (size_t)(p0 + (long long)i * pstep);
#pragma unroll
            for (int w = 0; w < KW; ++w) Cw[w] = scale_cost<WRAP>(cb[j][w], k.costScale);
            const int curI = ib[j];
            if (i == 0) {
#pragma unroll
                for (int w = 0; w < KW; ++w) Ln[w] = Cw[w] | mk.padMask[w];
            } else {
                const int p2 = p2lut[abs(curI - prevI)];
                sgm_step<KW, WRAP, FULL>(Lp, Cw, minPrev, p2, k.p1x2, k.bsub, mk, Ln);
            }
            prevI = curI;
            uint16_t* ap = pv.agg + p * Dp + off;
            if (first) {
                store_words<KW>(ap, Ln);
            } else {
                uint32_t a[KW];
#pragma unroll
                for (int w = 0; w < KW; ++w) a[w] = WRAP ? __vadd2(ab[j][w], Ln[w]) : ab[j][w] + Ln[w];
                store_words<KW>(ap, a);
            }
            // prefetch pixel i + PF into this slot
            if (i + PF < len) {
                const size_t q = (size_t)(p0 + (long long)(i + PF) * pstep);
                load_cost_words<KW>(pv.cost + q * Dp + off, cb[j]);
                if (!first) load_words<KW>(pv.agg + q * Dp + off, ab[j]);
                ib[j] = pv.img[q];
            }
#pragma unroll
            for (int w = 0; w < KW; ++w) Lp[w] = Ln[w];
            minPrev = warp_min_u16<KW>(Lp);
        }
    }
}

template <int KW, bool WRAP, bool FULL>
static cudaError_t launch_dir_t(const PairView& pv, const SgmConsts& k, int dir, int first,
                                cudaStream_t s) {
    const int lines = num_lines(dir, k.W, k.H);
    const int warpsPerBlock = 4;
    const int grid = (lines + warpsPerBlock - 1) / warpsPerBlock;
    constexpr int PF = KW <= 4 ? 4 : 2;
    agg_dir_kernel<KW, WRAP, FULL, PF><<<grid, 32 * warpsPerBlock, 0, s>>>(pv, k, dir, first);
    return cudaGetLastError();
}

template <int KW>
static cudaError_t launch_dir_kw(const PairView& pv, const SgmConsts& k, int dir, int first,
                                 bool wrap, cudaStream_t s) {
    const bool full = (k.D == k.Dp);
    if (wrap) return full ? launch_dir_t<KW, true, true>(pv, k, dir, first, s)
                          : launch_dir_t<KW, true, false>(pv, k, dir, first, s);
    return full ? launch_dir_t<KW, false, true>(pv, k, dir, first, s)
                : launch_dir_t<KW, false, false>(pv, k, dir, first, s);
}

cudaError_t launch_aggregate_per_direction(const PairView& pv, const SgmConsts& k,
                                           unsigned pathMask, bool wrap, cudaStream_t s) {
    const int KW = k.Dp / 64;
    bool first = true;
    for (int dir = 0; dir < 8; ++dir) {
        if (!(pathMask & (1u << dir))) continue;
        cudaError_t e;
        switch (KW) {
        case 1: e = launch_dir_kw<1>(pv, k, dir, first, wrap, s); break;
        case 2: e = launch_dir_kw<2>(pv, k, dir, first, wrap, s); break;
        case 3: e = launch_dir_kw<3>(pv, k, dir, first, wrap, s); break;
        case 4: e = launch_dir_kw<4>(pv, k, dir, first, wrap, s); break;
        case 5: e = launch_dir_kw<5>(pv, k, dir, first, wrap, s); break;
        case 6: e = launch_dir_kw<6>(pv, k, dir, first, wrap, s); break;
        case 7: e = launch_dir_kw<7>(pv, k, dir, first, wrap, s); break;
        case 8: e = launch_dir_kw<8>(pv, k, dir, first, wrap, s); break;
        default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        first = false;
    }
    return cudaSuccess;
}

}  // namespace lumen
