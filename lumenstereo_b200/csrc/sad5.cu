// sad5.cu -- SAD cost volume for the default 5x5 window (blockSize 5).
//
// Same values as the reference's computeCostSAD (src/sgbm_kernels.cu:70-212):
// cost(x, y, d) = sum / count over the 5x5 window's valid cells of
// |Lf(x', y') - Rf(x' - minD - d, y')| (a cell is valid when x', y' and the
// matched right column lie in the image), integer division, 255 when no cell
// is valid; entries d >= D of the padded volume are 0.
//
// A CTA owns 64 output columns x kS5WY output rows and every disparity.  It
// works in batches of RB rows:
//  * column phase -- a unit (tile column c of the 64 plus a 2-column apron on
//    each side, group g of 16 disparities) keeps the group's vertical 5-row
//    sums in registers as eight uint16x2 words (disparity pairs (d, d+2) and
//    (d+1, d+3) of every quad) and slides them down one row at a time: one
//    __vabsdiffu4 per quad for the entering row and one for the leaving row;
//    after each row it stores the sums to shared memory (RB snapshots);
//  * window phase -- a unit (row of the batch, run of 8 output columns,
//    group g) adds the five column sums of its first column and slides along
//    the run (one column in, one out), divides by the window count with one
//    multiply-high per value (umulhi(sum, ceil(2^32 / count)), exact for every
//    reachable sum) and writes the group's 16 cost bytes with one 16-byte
//    store.  A run whose window is whole for every output and every
//    disparity of the group (the interior) takes the count 25 without any
//    per-value test.
// Image rows are staged in a ring of RB + 5 rows; the right rows reversed
// (disparity ascending = address ascending) in four copies shifted by 0..3
// bytes, so every quad of disparities is one aligned 32-bit load.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

constexpr int kS5WX = 64;                 // output columns per CTA
constexpr int kS5WY = 32;                 // output rows per CTA
constexpr int kS5WC = kS5WX + 4;          // tile columns with the 2-column aprons
constexpr int kS5WCP = 80;                // staged left-row bytes (kS5WC rounded up to 16)

// rows per batch: RB * KP = 8 keeps the window phase at 256 units for Dp <= 256
__host__ __device__ constexpr int s5w_rb(int KP) { return KP <= 1 ? 8 : KP == 2 ? 4 : KP <= 4 ? 2 : 1; }
__host__ __device__ constexpr int s5w_rspan(int KP) { return (kS5WC + 64 * KP + 4 + 15) & ~15; }
__host__ __device__ constexpr size_t s5w_smem(int KP) {
    return (size_t)(s5w_rb(KP) + 5) * (kS5WCP + 4 * s5w_rspan(KP)) +           // staged rows
           (size_t)s5w_rb(KP) * kS5WC * 64 * KP * 2;                             // column sums
}

// Cost bytes of one quad (d0 .. d0+3) at column x outside the interior: the
// window's count from its valid rows (cy) and columns, 255 with none, 0 for
// d >= D.  ev = sums of (d0, d0+2), od = of (d0+1, d0+3).
__device__ __noinline__ uint32_t sad5w_edge_quad(uint32_t ev, uint32_t od, int d0, int x, int cy, int W, int D,
                                                int minD, const uint32_t* __restrict__ magic) {
    const uint32_t sv[4] = {ev & 0xFFFFu, od & 0xFFFFu, ev >> 16, od >> 16};
    uint32_t ow = 0;
#pragma unroll
    for (int bb = 0; bb < 4; ++bb) {
        const int d = d0 + bb;
        uint32_t v;
        if (d >= D) {
            v = 0;
        } else {
            const int ad = minD + d;
            const int clo = max(max(-2, -x), ad - x);
            const int chi = min(2, W - 1 - x);
            const int cnt = cy * max(0, chi - clo + 1);
            v = cnt > 0 ? (cnt == 1 ? sv[bb] : __umulhi(sv[bb], magic[cnt])) : 255u;
        }
        ow |= v << (8 * bb);
    }
    return ow;
}

template <int KP>
__global__ void __launch_bounds__(256)
sad5w_kernel(const uint8_t* __restrict__ pl, const uint8_t* __restrict__ pr, int W, int H, int D,
             int minD, const uint32_t* __restrict__ magic, uint8_t* __restrict__ cost) {
    constexpr int Dp = 64 * KP, KG = Dp / 16, RB = s5w_rb(KP), NR = RB + 5;
    constexpr int RS = s5w_rspan(KP);
    constexpr int CU = (kS5WC * KG + 255) / 256;      // column units per thread
    extern __shared__ __align__(16) uint8_t sm[];
    uint8_t* sL = sm;                                  // [NR][kS5WCP]
    uint8_t* sR = sL + NR * kS5WCP;                    // [NR][4][RS]
    uint4* csm = reinterpret_cast<uint4*>(sR + NR * 4 * RS);  // [RB][kS5WC][KG][2]
    const int x0 = blockIdx.x * kS5WX, y0 = blockIdx.y * kS5WY;
    const int yEnd = min(H, y0 + kS5WY);
    const int lx0 = x0 - 2;                            // image column of tile column 0
    const int rtop = lx0 + kS5WC - 1 - minD;           // right column at reversed index 0
    const int tid = threadIdx.x;

    auto stage_row = [&](int gy) {
        const int slot = gy % NR;
        for (int i = tid; i < kS5WCP; i += 256) {
            const int gx = lx0 + i;
            sL[slot * kS5WCP + i] = (i < kS5WC && gx >= 0 && gx < W) ? pl[(size_t)gy * W + gx] : 0;
        }
        for (int i = tid; i < 4 * RS; i += 256) {
            const int k = i / RS, j = i - k * RS;
            const int gx = rtop - (j + k);
            sR[(slot * 4 + k) * RS + j] = (gx >= 0 && gx < W) ? pr[(size_t)gy * W + gx] : 0;
        }
    };

    // ---- column units: (tile column c, group g); masks of valid bytes per quad ----
    int ucol[CU], ugrp[CU];
    uint32_t umask[CU][4];
#pragma unroll
    for (int k = 0; k < CU; ++k) {
        const int u = tid + 256 * k;
        const int c = u / KG, g = u - c * KG;
        ucol[k] = u < kS5WC * KG ? c : -1;
        ugrp[k] = g;
        const int xg = lx0 + c;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t m = 0;
            if (ucol[k] >= 0 && xg >= 0 && xg < W) {
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int d = 16 * g + 4 * q + b;
                    if (d < D && xg - minD - d >= 0) m |= 0xFFu << (8 * b);
                }
            }
            umask[k][q] = m;
        }
    }
    // A of one staged row for unit k, quad q: (d, d+2) and (d+1, d+3) uint16x2 words
    auto absdiff = [&](int slot, int k, int q, uint32_t& ev, uint32_t& od) {
        const int c = ucol[k];
        const uint32_t l4 = (uint32_t)sL[slot * kS5WCP + c] * 0x01010101u;
        const int j0 = (kS5WC - 1 - c) + 16 * ugrp[k] + 4 * q;
        const uint32_t r4 = *reinterpret_cast<const uint32_t*>(sR + (slot * 4 + (j0 & 3)) * RS + (j0 & ~3));
        const uint32_t v = __vabsdiffu4(l4, r4) & umask[k][q];
        ev = v & 0x00FF00FFu;
        od = (v >> 8) & 0x00FF00FFu;
    };

    uint32_t sE[CU][4], sO[CU][4];
    // the first batch's rows: y0-2 .. y0+RB+1 (y0-3 is never needed at y0)
    for (int gy = max(0, y0 - 2); gy <= min(H - 1, y0 + RB + 1); ++gy) stage_row(gy);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < CU; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            sE[k][q] = 0;
            sO[k][q] = 0;
            if (ucol[k] >= 0)
                for (int gy = max(0, y0 - 2); gy <= min(H - 1, y0 + 2); ++gy) {
                    uint32_t e, o;
                    absdiff(gy % NR, k, q, e, o);
                    sE[k][q] += e;
                    sO[k][q] += o;
                }
        }

    // ---- window units: (row of the batch, run of 8 columns, group g) ----
    const int wg = tid % KG, wrest = tid / KG;
    const int wk = wrest % (kS5WX / 8), wrb = wrest / (kS5WX / 8);
    const bool wOn = wrb < RB;
    const int px0 = 8 * wk;                            // first output column of the run (tile)
    const int xr0 = x0 + px0;                          // its image column
    const int dg0 = 16 * wg;
    // the run's windows are whole in x, and every disparity of the group is matched inside
    const bool xInterior = xr0 - 2 >= 0 && xr0 + 7 + 2 <= W - 1 && xr0 - 2 - minD - (dg0 + 15) >= 0 &&
                           dg0 + 16 <= D;
    const uint32_t m25 = magic[25];

    for (int yb = y0; yb < yEnd; yb += RB) {
        if (yb > y0) {
            // entering rows of this batch: yb+2 .. yb+RB+1
            __syncthreads();  // the previous batch's column phase is done with the ring slots
            for (int gy = yb + 2; gy <= min(H - 1, yb + RB + 1); ++gy) stage_row(gy);
            __syncthreads();
        }
        // ---- column phase: RB rows ----
#pragma unroll 1
        for (int rb = 0; rb < RB; ++rb) {
            const int y = yb + rb;
            if (y >= yEnd) break;
            if (y > y0) {
                const int yin = y + 2, yout = y - 3;
                const bool hasIn = yin < H, hasOut = yout >= 0;
#pragma unroll
                for (int k = 0; k < CU; ++k) {
                    if (ucol[k] < 0) continue;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        uint32_t e, o;
                        if (hasIn) {
                            absdiff(yin % NR, k, q, e, o);
                            sE[k][q] += e;
                            sO[k][q] += o;
                        }
                        if (hasOut) {
                            absdiff(yout % NR, k, q, e, o);
                            sE[k][q] -= e;
                            sO[k][q] -= o;
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < CU; ++k) {
                if (ucol[k] < 0) continue;
                uint4* dst = csm + ((size_t)(rb * kS5WC + ucol[k]) * KG + ugrp[k]) * 2;
                dst[0] = make_uint4(sE[k][0], sO[k][0], sE[k][1], sO[k][1]);
                dst[1] = make_uint4(sE[k][2], sO[k][2], sE[k][3], sO[k][3]);
            }
        }
        __syncthreads();
        // ---- window phase ----
        const int y = yb + wrb;
        if (wOn && y < yEnd) {
            const int cy = min(H - 1, y + 2) - max(0, y - 2) + 1;   // valid window rows
            const uint4* col = csm + ((size_t)(wrb * kS5WC) * KG + wg) * 2;   // column 0 of this group
            uint32_t acc[8];
#pragma unroll
            for (int w = 0; w < 8; ++w) acc[w] = 0;
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const uint4 a = col[(size_t)(px0 + c) * KG * 2], b = col[(size_t)(px0 + c) * KG * 2 + 1];
                acc[0] += a.x; acc[1] += a.y; acc[2] += a.z; acc[3] += a.w;
                acc[4] += b.x; acc[5] += b.y; acc[6] += b.z; acc[7] += b.w;
            }
            const bool interior = xInterior && cy == 5;
            uint8_t* out = cost + ((size_t)y * W + xr0) * Dp + dg0;
#pragma unroll 1
            for (int i = 0; i < 8; ++i) {
                if (i > 0) {
                    const uint4 a = col[(size_t)(px0 + i + 4) * KG * 2], b = col[(size_t)(px0 + i + 4) * KG * 2 + 1];
                    const uint4 e = col[(size_t)(px0 + i - 1) * KG * 2], f = col[(size_t)(px0 + i - 1) * KG * 2 + 1];
                    acc[0] += a.x - e.x; acc[1] += a.y - e.y; acc[2] += a.z - e.z; acc[3] += a.w - e.w;
                    acc[4] += b.x - f.x; acc[5] += b.y - f.y; acc[6] += b.z - f.z; acc[7] += b.w - f.w;
                }
                const int x = xr0 + i;
                if (x >= W) break;
                uint32_t o4[4];
                if (interior) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        // acc[2q] = (d, d+2), acc[2q+1] = (d+1, d+3) of quad q
                        const uint32_t ev = acc[2 * q], od = acc[2 * q + 1];
                        const uint32_t qe = __umulhi(ev & 0xFFFFu, m25) + (__umulhi(ev >> 16, m25) << 16);
                        const uint32_t qo = __umulhi(od & 0xFFFFu, m25) + (__umulhi(od >> 16, m25) << 16);
                        o4[q] = qe + (qo << 8);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) o4[q] = sad5w_edge_quad(acc[2 * q], acc[2 * q + 1], dg0 + 4 * q, x, cy, W, D, minD, magic);
                }
                *reinterpret_cast<uint4*>(out + (size_t)i * Dp) = make_uint4(o4[0], o4[1], o4[2], o4[3]);
            }
        }
    }
}

template <int KP>
static cudaError_t launch_sad5w_kp(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int minD,
                                   const uint32_t* magic, uint8_t* cost, cudaStream_t s) {
    const size_t smem = s5w_smem(KP);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(sad5w_kernel<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 g((W + kS5WX - 1) / kS5WX, (H + kS5WY - 1) / kS5WY);
    sad5w_kernel<KP><<<g, 256, smem, s>>>(pl, pr, W, H, D, minD, magic, cost);
    return cudaGetLastError();
}

// The 5x5 window (r = 2) for padded disparity counts up to 448; cudaErrorInvalidValue otherwise.
cudaError_t launch_sad5w(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int Dp, int minD,
                         const uint32_t* magic, uint8_t* cost, cudaStream_t s) {
    switch (Dp / 64) {
    case 1: return launch_sad5w_kp<1>(pl, pr, W, H, D, minD, magic, cost, s);
    case 2: return launch_sad5w_kp<2>(pl, pr, W, H, D, minD, magic, cost, s);
    case 3: return launch_sad5w_kp<3>(pl, pr, W, H, D, minD, magic, cost, s);
    case 4: return launch_sad5w_kp<4>(pl, pr, W, H, D, minD, magic, cost, s);
    case 5: return launch_sad5w_kp<5>(pl, pr, W, H, D, minD, magic, cost, s);
    case 6: return launch_sad5w_kp<6>(pl, pr, W, H, D, minD, magic, cost, s);
    case 7: return launch_sad5w_kp<7>(pl, pr, W, H, D, minD, magic, cost, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace lumen
