// cost.cu -- input staging, prefilter, census and the uint8 cost volumes.
//
// Volume layout: cost[(y*W + x)*Dp + d], d fastest, Dp = D rounded up to 64;
// entries d >= D are 0.  Values for d < D equal the reference's:
//   SAD    src/sgbm_kernels.cu:70-212   integer mean of |Lf-Rf| over the valid
//                                       part of the window, 255 if none valid
//   Census src/sgbm_kernels.cu:250-286  (h*255+12)/24, 255 in the 2-px border
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace lumen {

// ---------------------------------------------------------------------------
// Input staging: gray copy (channels == 1) or BGR -> gray (channels == 3) of
// both images into pitch-W buffers.  BGR uses BT.601 in 15-bit fixed point,
// Y = (3735 B + 19235 G + 9798 R + 16384) >> 15, the 8-bit path of
// cv::cvtColor(COLOR_BGR2GRAY) (OpenCV 4.x) that the reference runs on the
// host (src/sgbm_gpu.cu:169-172).
// ---------------------------------------------------------------------------
__global__ void stage_gray_kernel(const uint8_t* __restrict__ l, const uint8_t* __restrict__ r,
                                  size_t pitch, int channels, int W, int H,
                                  uint8_t* __restrict__ gl, uint8_t* __restrict__ gr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const uint8_t* src = blockIdx.z ? r : l;
    uint8_t* dst = blockIdx.z ? gr : gl;
    if (x >= W) return;
    const uint8_t* row = src + (size_t)y * pitch;
    uint8_t v;
    if (channels == 1) {
        v = row[x];
    } else {
        const int b = row[3 * x], g = row[3 * x + 1], rr = row[3 * x + 2];
        v = (uint8_t)((3735 * b + 19235 * g + 9798 * rr + 16384) >> 15);
    }
    dst[(size_t)y * W + x] = v;
}

// src/sgbm_kernels.cu:38-59 (prefilterXSobel) for both images.
__global__ void prefilter_kernel(const uint8_t* __restrict__ gl, const uint8_t* __restrict__ gr,
                                 int W, int H, int cap, uint8_t* __restrict__ pl,
                                 uint8_t* __restrict__ pr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const uint8_t* row = (blockIdx.z ? gr : gl) + (size_t)y * W;
    int val;
    if (x > 0 && x < W - 1) val = (int)row[x + 1] - (int)row[x - 1];
    else if (x == 0) val = (int)row[1] - (int)row[0];
    else val = (int)row[x] - (int)row[x - 1];
    val = min(cap, max(-cap, val));
    (blockIdx.z ? pr : pl)[(size_t)y * W + x] = (uint8_t)(val + cap);
}

// src/sgbm_kernels.cu:217-245 (buildCensus5x5) for both images; a 16x16 tile
// with a 2-pixel apron staged in shared memory.
__global__ void census_kernel(const uint8_t* __restrict__ gl, const uint8_t* __restrict__ gr,
                              int W, int H, uint32_t* __restrict__ cl, uint32_t* __restrict__ cr) {
    __shared__ uint8_t tile[20][21];
    const uint8_t* img = blockIdx.z ? gr : gl;
    uint32_t* out = blockIdx.z ? cr : cl;
    const int bx = blockIdx.x * 16, by = blockIdx.y * 16;
    for (int i = threadIdx.y * 16 + threadIdx.x; i < 20 * 20; i += 256) {
        const int ty = i / 20, tx = i % 20;
        const int gx = bx + tx - 2, gy = by + ty - 2;
        tile[ty][tx] = (gx >= 0 && gx < W && gy >= 0 && gy < H) ? img[(size_t)gy * W + gx] : 0;
    }
    __syncthreads();
    const int x = bx + threadIdx.x, y = by + threadIdx.y;
    if (x >= W || y >= H) return;
    uint32_t bits = 0u;
    if (!(x < 2 || x >= W - 2 || y < 2 || y >= H - 2)) {
        const uint8_t c = tile[threadIdx.y + 2][threadIdx.x + 2];
        int bit = 0;
#pragma unroll
        for (int dy = 0; dy < 5; ++dy)
#pragma unroll
            for (int dx = 0; dx < 5; ++dx) {
                if (dx == 2 && dy == 2) continue;
                bits |= (uint32_t)(tile[threadIdx.y + dy][threadIdx.x + dx] >= c) << bit;
                ++bit;
            }
    }
    out[(size_t)y * W + x] = bits;
}

// (h*255+12)/24 == (85*h+4)>>3 for every h in [0,24] (255h+12 = 3(85h+4)).
__device__ __forceinline__ uint32_t census_cost_of(int h) { return (uint32_t)((85 * h + 4) >> 3); }

// src/sgbm_kernels.cu:250-286 (computeCostCensus_naive).  One CTA per (row,
// 128-pixel tile).  The tile's left descriptors and every right descriptor it
// can reach are staged in shared memory; a thread takes 4 consecutive pixels
// x 16 consecutive disparities and reads the 19 right descriptors that block
// reaches as five aligned 16-byte loads (right column x - d for pixel i,
// disparity dlo + k is window word 15 + i - k).  Blocks whose pixels and
// right columns all lie inside the 2-px border convert two Hamming distances
// per instruction, ((85*(h0 | h1<<16) + 0x40004) >> 3) & 0x00FF00FF; the
// others take the per-disparity border rules.  The tile's costs go through
// shared memory (rows padded so the 16-byte writes of a quarter-warp hit
// distinct banks) and leave as contiguous 16-byte stores.
constexpr int kCensusTile = 128;
constexpr int kCensusPx = 4;   // consecutive pixels a thread

// shared-memory words: left descriptors, right descriptors, cost tile
__host__ __device__ inline int census_tile_pitch_words(int Dp) {
    const int w = Dp / 4;
    return w % 8 == 0 ? w + 4 : w;   // an odd multiple of 4 words between rows
}
__host__ __device__ inline int census_right_words(int Dp) { return kCensusTile + Dp + 4; }
__host__ __device__ inline size_t census_smem_bytes(int Dp) {
    return 4 * ((size_t)kCensusTile + census_right_words(Dp) + (size_t)kCensusTile * census_tile_pitch_words(Dp));
}

__global__ void __launch_bounds__(256)
census_cost_kernel(const uint32_t* __restrict__ cl, const uint32_t* __restrict__ cr, int W,
                   int H, int D, int Dp, int minD, uint8_t* __restrict__ cost) {
    extern __shared__ __align__(16) uint32_t sm_c[];
    uint32_t* const sl = sm_c;                       // kCensusTile left descriptors
    uint32_t* const sr = sm_c + kCensusTile;         // right descriptors of columns lo, lo+1, ...
    const int RW = census_right_words(Dp);
    const int P = census_tile_pitch_words(Dp);
    uint32_t* const tile = sr + RW;                  // costs, pixel p at word p * P
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * kCensusTile;
    const int lo = x0 - minD - (Dp - 1);             // right column of sr[0]
    for (int i = threadIdx.x; i < RW; i += blockDim.x) {
        const int rx = lo + i;
        sr[i] = (rx >= 0 && rx < W) ? cr[(size_t)y * W + rx] : 0u;
    }
    for (int i = threadIdx.x; i < kCensusTile; i += blockDim.x) {
        const int x = x0 + i;
        sl[i] = x < W ? cl[(size_t)y * W + x] : 0u;
    }
    __syncthreads();
    const int chunks = Dp / 16;
    const bool rowOk = y >= 2 && y < H - 2;
    constexpr int groups = kCensusTile / kCensusPx;
    // item -> (pixel group pg, chunk ch), pg fastest: a quarter-warp's window
    // loads cover 128 contiguous bytes
    for (int it = threadIdx.x; it < groups * chunks; it += blockDim.x) {
        const int pg = it % groups, ch = it / groups;
        const int xb = x0 + pg * kCensusPx;
        if (xb >= W) continue;
        const int dlo = ch * 16;
        const int rxTop = xb + kCensusPx - 1 - minD - dlo;   // right column of (pixel 3, dlo)
        uint8_t* const out = reinterpret_cast<uint8_t*>(tile) + (size_t)pg * kCensusPx * P * 4 + dlo;
        const bool fast = rowOk && xb >= 2 && xb + kCensusPx - 1 < W - 2 && rxTop - 18 >= 2 &&
                          rxTop < W - 2 && dlo + 16 <= D;
        if (fast) {
            // window word m holds right column rxTop - 18 + m; its index in sr is a
            // multiple of 4 (pg*4 - dlo + Dp - 16)
            uint32_t w[20];
            const uint4* wp = reinterpret_cast<const uint4*>(sr + (rxTop - 18 - lo));
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const uint4 v = wp[q];
                w[4 * q] = v.x; w[4 * q + 1] = v.y; w[4 * q + 2] = v.z; w[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int i = 0; i < kCensusPx; ++i) {
                const uint32_t a = sl[pg * kCensusPx + i];
                uint32_t wv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t h0 = __popc(a ^ w[15 + i - (4 * q + 0)]);
                    const uint32_t h1 = __popc(a ^ w[15 + i - (4 * q + 1)]);
                    const uint32_t h2 = __popc(a ^ w[15 + i - (4 * q + 2)]);
                    const uint32_t h3 = __popc(a ^ w[15 + i - (4 * q + 3)]);
                    const uint32_t c02 = ((85u * (h0 | (h2 << 16)) + 0x40004u) >> 3) & 0x00FF00FFu;
                    const uint32_t c13 = ((85u * (h1 | (h3 << 16)) + 0x40004u) >> 3) & 0x00FF00FFu;
                    wv[q] = c02 | (c13 << 8);
                }
                *reinterpret_cast<uint4*>(out + (size_t)i * P * 4) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < kCensusPx; ++i) {
                const int x = xb + i;
                const bool leftOk = rowOk && x >= 2 && x < W - 2;
                const uint32_t a = leftOk ? sl[pg * kCensusPx + i] : 0u;
                uint32_t wv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t packed = 0;
#pragma unroll
                    for (int bb = 0; bb < 4; ++bb) {
                        const int d = dlo + q * 4 + bb;
                        const int rx = x - minD - d;
                        uint32_t c;
                        if (d >= D) c = 0u;
                        else if (!leftOk || rx < 2 || rx >= W - 2) c = 255u;
                        else c = census_cost_of(__popc(a ^ sr[rx - lo]));
                        packed |= c << (8 * bb);
                    }
                    wv[q] = packed;
                }
                *reinterpret_cast<uint4*>(out + (size_t)i * P * 4) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            }
        }
    }
    __syncthreads();
    // the tile's rows, contiguous in the volume, as 16-byte stores
    const int npx = min(kCensusTile, W - x0);
    const int cpr = Dp / 16;                         // 16-byte chunks a pixel
    uint8_t* const dst = cost + ((size_t)y * W + x0) * Dp;
    for (int c = threadIdx.x; c < npx * cpr; c += blockDim.x) {
        const int px = c / cpr, k = c - px * cpr;
        const uint4 v = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint8_t*>(tile) +
                                                        (size_t)px * P * 4 + 16 * k);
        *reinterpret_cast<uint4*>(dst + (size_t)c * 16) = v;
    }
}

// ---------------------------------------------------------------------------
// SAD cost (src/sgbm_kernels.cu:70-212).
//
// One CTA per (64-pixel column tile, band of kSadBand rows), sliding down the
// band.  Shared memory keeps, per column x' of the tile plus an r-pixel apron
// and per 4-disparity quad, the column sums
//   cs[x'][d] = sum over the window's valid rows of A(x', row, d),
//   A = |Lf(x',row) - Rf(x'-ad,row)| (0 when x' or x'-ad is outside the image),
// four disparities per __vabsdiffu4, stored as two uint16x2 words holding
// (d0,d2) and (d1,d3).  Moving one row down adds the entering row and
// subtracts the leaving one (rows are kept in a small ring), so every A value
// is computed twice instead of 2r+1 times.  Window sums then slide along x
// (add the entering column, subtract the leaving one).  The count is
// (#valid rows) x (#valid columns) and sum/count = umulhi(sum, ceil(2^32/count)),
// exact for every reachable sum.  WIDE keeps 32-bit window sums when
// (2r+1)^2 * 2*cap can exceed 65535.
// ---------------------------------------------------------------------------
constexpr int kSadTile = 64;   // output columns per CTA
constexpr int kSadBand = 32;   // output rows per CTA
constexpr int kSadRun = 8;     // consecutive output pixels per thread (window sliding)

struct SadGeom {
    int nrow;   // 2r+1
    int ncol;   // kSadTile + 2r
    int ncolp;  // ncol rounded up to 4
    int rw;     // reversed right-row span (bytes), multiple of 4
    int ring;   // rows kept: 2r+2
};

__host__ __device__ inline SadGeom sad_geom(int Dp, int r) {
    SadGeom g;
    g.nrow = 2 * r + 1;
    g.ncol = kSadTile + 2 * r;
    g.ncolp = (g.ncol + 3) & ~3;
    g.rw = (g.ncol + Dp - 1 + 3 + 4) & ~3;
    g.ring = 2 * r + 2;
    return g;
}

__device__ __forceinline__ uint32_t load_u32_unaligned(const uint8_t* base, int i) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(base + (i & ~3));
    return __byte_perm(w[0], w[1], (uint32_t)(0x3210 + 0x1111 * (i & 3)));
}

// abs differences of one row for column c and the quad d0..d0+3, split as
// (d0,d2) / (d1,d3) uint16x2 words.
__device__ __forceinline__ void sad_row_quad(const uint8_t* sLrow, const uint8_t* sRrow, int c,
                                             int j0, uint32_t mask, uint32_t& ev, uint32_t& od) {
    const uint32_t l4 = __byte_perm((uint32_t)sLrow[c], 0u, 0x0000);
    const uint32_t r4 = load_u32_unaligned(sRrow, j0);
    const uint32_t v = __vabsdiffu4(l4, r4) & mask;
    ev = v & 0x00FF00FFu;
    od = (v >> 8) & 0x00FF00FFu;
}

template <bool WIDE, int KP>
__global__ void __launch_bounds__(256)
sad_cost_kernel(const uint8_t* __restrict__ pl, const uint8_t* __restrict__ pr, int W, int H,
                int D, int minD, int r, const uint32_t* __restrict__ magic,
                uint8_t* __restrict__ cost) {
    constexpr int Dp = 64 * KP;  // padded disparities: divisions below are by constants
    extern __shared__ __align__(16) uint8_t sm[];
    const SadGeom g = sad_geom(Dp, r);
    const int x0 = blockIdx.x * kSadTile;
    const int yb = blockIdx.y * kSadBand;
    const int yEnd = min(H, yb + kSadBand);
    const int lx0 = x0 - r;                        // column of cs index 0
    const int rtop = lx0 + g.ncol - 1 - minD;      // right column at reversed index 0
    constexpr int quads = Dp / 4;
    uint8_t* sL = sm;                              // [ring][ncolp]
    uint8_t* sR = sL + g.ring * g.ncolp;           // [ring][rw]
    uint2* cs = reinterpret_cast<uint2*>(sm + ((g.ring * (g.ncolp + g.rw) + 15) & ~15));  // [ncol][quads]

    auto load_row = [&](int gy) {  // row gy into ring slot gy % ring
        const int slot = gy % g.ring;
        for (int i = threadIdx.x; i < g.ncolp; i += blockDim.x) {
            const int gx = lx0 + i;
            sL[slot * g.ncolp + i] = (gx >= 0 && gx < W && i < g.ncol) ? pl[(size_t)gy * W + gx] : 0;
        }
        for (int j = threadIdx.x; j < g.rw; j += blockDim.x) {
            const int gx = rtop - j;
            sR[slot * g.rw + j] = (gx >= 0 && gx < W) ? pr[(size_t)gy * W + gx] : 0;
        }
    };
    // validity mask of (column c, quad q): bytes whose column and right pixel are in the image
    auto quad_mask = [&](int c, int q) -> uint32_t {
        const int xg = lx0 + c;
        if (xg < 0 || xg >= W) return 0u;
        const int d0 = 4 * q;
        const int rx0 = xg - minD - d0;  // right column of byte 0; byte b: rx0 - b
        if (rx0 - 3 >= 0 && rx0 < W && d0 + 4 <= D) return 0xFFFFFFFFu;
        uint32_t m = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b)
            if (rx0 - b >= 0 && rx0 - b < W && d0 + b < D) m |= 0xFFu << (8 * b);
        return m;
    };

    // initial window rows of the first output row
    for (int gy = max(0, yb - r); gy <= min(H - 1, yb + r); ++gy) load_row(gy);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int c = warp; c < g.ncol; c += nw) {
        for (int q = lane; q < quads; q += 32) {
            const uint32_t mask = quad_mask(c, q);
            const int j0 = rtop - (lx0 + c - minD - 4 * q);
            uint32_t ev = 0, od = 0;
            if (mask)
                for (int gy = max(0, yb - r); gy <= min(H - 1, yb + r); ++gy) {
                    uint32_t e, o;
                    const int slot = gy % g.ring;
                    sad_row_quad(sL + slot * g.ncolp, sR + slot * g.rw, c, j0, mask, e, o);
                    ev += e;
                    od += o;
                }
            cs[c * quads + q] = make_uint2(ev, od);
        }
    }
    for (int y = yb; y < yEnd; ++y) {
        if (y > yb) {
            // slide: add row y+r, remove row y-r-1
            const int yin = y + r, yout = y - r - 1;
            if (yin < H) load_row(yin);
            __syncthreads();
            const bool hasIn = yin < H, hasOut = yout >= 0;
            const uint8_t* sLin = sL + (hasIn ? yin % g.ring : 0) * g.ncolp;
            const uint8_t* sRin = sR + (hasIn ? yin % g.ring : 0) * g.rw;
            const uint8_t* sLout = sL + (hasOut ? yout % g.ring : 0) * g.ncolp;
            const uint8_t* sRout = sR + (hasOut ? yout % g.ring : 0) * g.rw;
            for (int c = warp; c < g.ncol; c += nw) {
#pragma unroll
                for (int q = lane; q < quads; q += 32) {
                    const uint32_t mask = quad_mask(c, q);
                    if (!mask) continue;
                    const int j0 = rtop - (lx0 + c - minD - 4 * q);
                    uint2 v = cs[c * quads + q];
                    uint32_t e, o;
                    if (hasIn) {
                        sad_row_quad(sLin, sRin, c, j0, mask, e, o);
                        v.x += e;
                        v.y += o;
                    }
                    if (hasOut) {
                        sad_row_quad(sLout, sRout, c, j0, mask, e, o);
                        v.x -= e;
                        v.y -= o;
                    }
                    cs[c * quads + q] = v;
                }
            }
        }
        __syncthreads();
        // window sums: thread -> (quad, run of kSadRun pixels)
        const int cy = min(H - 1, y + r) - max(0, y - r) + 1;
        const int full = cy * (2 * r + 1);
        const uint32_t mfull = magic[full];
        const int runs = kSadTile / kSadRun;
        for (int item = threadIdx.x; item < quads * runs; item += blockDim.x) {
            const int q = item % quads, run = item / quads;  // quads is a compile-time constant
            const int px0 = run * kSadRun;
            const int d0 = 4 * q;
            uint32_t s0, s1, s2, s3;  // window sums of d0..d0+3 (WIDE) or packed pairs
            uint32_t pe = 0, po = 0;
            uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
            // columns of pixel px: cs index px .. px + 2r
            for (int k = 0; k < 2 * r + 1; ++k) {
                const uint2 v = cs[(px0 + k) * quads + q];
                if (WIDE) {
                    w0 += v.x & 0xFFFFu; w2 += v.x >> 16; w1 += v.y & 0xFFFFu; w3 += v.y >> 16;
                } else {
                    pe += v.x;
                    po += v.y;
                }
            }
            for (int t = 0; t < kSadRun; ++t) {
                const int px = px0 + t;
                const int x = x0 + px;
                if (t > 0) {
                    const uint2 vin = cs[(px + 2 * r) * quads + q];
                    const uint2 vout = cs[(px - 1) * quads + q];
                    if (WIDE) {
                        w0 += (vin.x & 0xFFFFu) - (vout.x & 0xFFFFu);
                        w2 += (vin.x >> 16) - (vout.x >> 16);
                        w1 += (vin.y & 0xFFFFu) - (vout.y & 0xFFFFu);
                        w3 += (vin.y >> 16) - (vout.y >> 16);
                    } else {
                        pe += vin.x - vout.x;
                        po += vin.y - vout.y;
                    }
                }
                if (x >= W) break;
                if (WIDE) { s0 = w0; s1 = w1; s2 = w2; s3 = w3; }
                else { s0 = pe & 0xFFFFu; s2 = pe >> 16; s1 = po & 0xFFFFu; s3 = po >> 16; }
                uint32_t outw;
                const bool interior = (x - r >= 0) && (x + r <= W - 1) && (x - r - minD - d0 - 3 >= 0) &&
                                      (d0 + 4 <= D);
                if (interior) {
                    const uint32_t q0 = full == 1 ? s0 : __umulhi(s0, mfull);
                    const uint32_t q1 = full == 1 ? s1 : __umulhi(s1, mfull);
                    const uint32_t q2 = full == 1 ? s2 : __umulhi(s2, mfull);
                    const uint32_t q3 = full == 1 ? s3 : __umulhi(s3, mfull);
                    outw = q0 | (q1 << 8) | (q2 << 16) | (q3 << 24);
                } else {
                    const uint32_t sv[4] = {s0, s1, s2, s3};
                    outw = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int d = d0 + b;
                        uint32_t v;
                        if (d >= D) {
                            v = 0;
                        } else {
                            const int ad = minD + d;
                            const int clo = max(max(-r, -x), ad - x);
                            const int chi = min(min(r, W - 1 - x), W - 1 - x + ad);
                            const int cnt = cy * max(0, chi - clo + 1);
                            v = cnt > 0 ? (cnt == 1 ? sv[b] : __umulhi(sv[b], magic[cnt])) : 255u;
                        }
                        outw |= v << (8 * b);
                    }
                }
                *reinterpret_cast<uint32_t*>(cost + ((size_t)y * W + x) * Dp + d0) = outw;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// SAD cost for the 5x5 window (blockSize 5, the default) and 16-bit sums.
//
// Same sums, counts and divisions as sad_cost_kernel; a leaner schedule.  A
// CTA owns 32 output columns x 32 output rows and all Dp disparities; thread
// (quad q, column lane cl) owns disparities 4q..4q+3 of the columns cl,
// cl + CLN, ... of the tile plus its 2-pixel apron.  It keeps their column
// sums (two uint16x2 words: d0,d2 / d1,d3) in registers and slides them down
// the rows: one __vabsdiffu4 for the entering row and one for the leaving
// row per column and quad.  The right rows are staged reversed (disparity
// ascending = address ascending) in four copies shifted by 0..3 bytes, so
// every quad is one aligned 32-bit load.  Column sums go through shared
// memory once per row; the window sums slide along x over a run of columns
// per thread, and the interior (full window, every disparity of the quad
// valid) divides by one constant per row.
// ---------------------------------------------------------------------------
constexpr int kS5X = 32;   // output columns per CTA
constexpr int kS5Y = 32;   // output rows per CTA
constexpr int kS5R = 2;    // window radius
constexpr int kS5C = kS5X + 2 * kS5R;  // columns with apron
constexpr int kS5Ring = 2 * kS5R + 2;  // staged rows

__host__ __device__ constexpr int s5_quads(int KP) { return 16 * KP; }
// column lanes per quad: the largest power of two with Q * CLN <= 256
__host__ __device__ constexpr int s5_cln(int KP) {
    return 256 / s5_quads(KP) >= 16 ? 16 : 256 / s5_quads(KP) >= 8 ? 8 : 256 / s5_quads(KP) >= 4 ? 4
         : 256 / s5_quads(KP) >= 2 ? 2 : 1;
}
__host__ __device__ constexpr int s5_rspan(int KP) { return (kS5C + 64 * KP + 3 + 4 + 15) & ~15; }

template <int KP>
__global__ void __launch_bounds__(256)
sad5_cost_kernel(const uint8_t* __restrict__ pl, const uint8_t* __restrict__ pr, int W, int H,
                 int D, int minD, const uint32_t* __restrict__ magic, uint8_t* __restrict__ cost) {
    constexpr int Dp = 64 * KP, Q = s5_quads(KP), CLN = s5_cln(KP);
    constexpr int NCOL = (kS5C + CLN - 1) / CLN;  // columns per thread (some idle at the end)
    constexpr int RUN = kS5X / CLN;               // output columns per thread
    constexpr int RS = s5_rspan(KP);              // reversed right-row span (bytes, per copy)
    static_assert(kS5X % CLN == 0, "runs tile the output columns");
    __shared__ __align__(16) uint8_t sL[kS5Ring][kS5C + 12];
    __shared__ __align__(16) uint8_t sR[kS5Ring][4][RS];
    __shared__ __align__(16) uint2 cs[kS5C][Q];
    const int x0 = blockIdx.x * kS5X, y0 = blockIdx.y * kS5Y;
    const int yEnd = min(H, y0 + kS5Y);
    const int q = threadIdx.x % Q, cl = threadIdx.x / Q;
    const int d0 = 4 * q;
    const int lx0 = x0 - kS5R;                 // image column of tile column 0
    const int rtop = lx0 + kS5C - 1 - minD;    // right column at reversed index 0
    const int nthreads = Q * CLN;

    auto stage_row = [&](int gy) {             // row gy into ring slot gy % kS5Ring
        const int slot = gy % kS5Ring;
        for (int i = threadIdx.x; i < kS5C; i += nthreads) {
            const int gx = lx0 + i;
            sL[slot][i] = (gx >= 0 && gx < W) ? pl[(size_t)gy * W + gx] : 0;
        }
        for (int i = threadIdx.x; i < 4 * RS; i += nthreads) {
            const int k = i / RS, j = i - k * RS;
            const int gx = rtop - (j + k);
            sR[slot][k][j] = (gx >= 0 && gx < W) ? pr[(size_t)gy * W + gx] : 0;
        }
    };
    // A of one row for tile column c: (d0,d2) and (d1,d3) as uint16x2 words
    auto absdiff = [&](int slot, int c, uint32_t mask, uint32_t& ev, uint32_t& od) {
        const uint32_t l4 = (uint32_t)sL[slot][c] * 0x01010101u;
        const int j0 = (kS5C - 1 - c) + d0;    // reversed index of (column c, d0)
        const uint32_t r4 = *reinterpret_cast<const uint32_t*>(&sR[slot][j0 & 3][j0 & ~3]);
        const uint32_t v = __vabsdiffu4(l4, r4) & mask;
        ev = v & 0x00FF00FFu;
        od = (v >> 8) & 0x00FF00FFu;
    };

    // column validity masks (per band: they depend on x and d only)
    uint32_t msk[NCOL];
#pragma unroll
    for (int i = 0; i < NCOL; ++i) {
        const int c = cl + i * CLN;
        const int xg = lx0 + c;
        uint32_t m = 0;
        if (c < kS5C && xg >= 0 && xg < W) {
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (xg - minD - (d0 + b) >= 0 && d0 + b < D) m |= 0xFFu << (8 * b);
        }
        msk[i] = m;
    }
    // initial column sums of the first output row
    for (int gy = max(0, y0 - kS5R); gy <= min(H - 1, y0 + kS5R); ++gy) stage_row(gy);
    __syncthreads();
    uint32_t cev[NCOL], cod[NCOL];
#pragma unroll
    for (int i = 0; i < NCOL; ++i) {
        cev[i] = 0;
        cod[i] = 0;
        const int c = cl + i * CLN;
        if (c < kS5C && msk[i])
            for (int gy = max(0, y0 - kS5R); gy <= min(H - 1, y0 + kS5R); ++gy) {
                uint32_t e, o;
                absdiff(gy % kS5Ring, c, msk[i], e, o);
                cev[i] += e;
                cod[i] += o;
            }
    }
    // output geometry of this thread's run
    const int px0 = cl * RUN;                 // first output column (tile-relative)
    for (int y = y0; y < yEnd; ++y) {
        if (y > y0) {
            // slide down: add row y + r, remove row y - r - 1 (both staged)
            const int yin = y + kS5R, yout = y - kS5R - 1;
            const bool hasIn = yin < H, hasOut = yout >= 0;
            const int sin = hasIn ? yin % kS5Ring : 0, sout = hasOut ? yout % kS5Ring : 0;
#pragma unroll
            for (int i = 0; i < NCOL; ++i) {
                const int c = cl + i * CLN;
                if (c < kS5C && msk[i]) {
                    uint32_t e, o;
                    if (hasIn) {
                        absdiff(sin, c, msk[i], e, o);
                        cev[i] += e;
                        cod[i] += o;
                    }
                    if (hasOut) {
                        absdiff(sout, c, msk[i], e, o);
                        cev[i] -= e;
                        cod[i] -= o;
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < NCOL; ++i) {
            const int c = cl + i * CLN;
            if (c < kS5C) cs[c][q] = make_uint2(cev[i], cod[i]);
        }
        __syncthreads();
        // stage the row the next step enters (its ring slot held row y - r - 1)
        if (y + 1 < yEnd && y + 1 + kS5R < H) stage_row(y + 1 + kS5R);
        // window sums along x, then counts and divisions
        const int cy = min(H - 1, y + kS5R) - max(0, y - kS5R) + 1;
        const int full = cy * (2 * kS5R + 1);
        const uint32_t mfull = magic[full];
        uint32_t pe = 0, po = 0;
#pragma unroll
        for (int k = 0; k < 2 * kS5R + 1; ++k) {
            const uint2 v = cs[px0 + k][q];
            pe += v.x;
            po += v.y;
        }
        uint8_t* crow = cost + ((size_t)y * W) * Dp + d0;
#pragma unroll
        for (int t = 0; t < RUN; ++t) {
            const int px = px0 + t;
            const int x = x0 + px;
            if (t > 0) {
                const uint2 vin = cs[px + 2 * kS5R][q];
                const uint2 vout = cs[px - 1][q];
                pe += vin.x - vout.x;
                po += vin.y - vout.y;
            }
            if (x < W) {
                const uint32_t s0 = pe & 0xFFFFu, s2 = pe >> 16, s1 = po & 0xFFFFu, s3 = po >> 16;
                uint32_t outw;
                const bool interior = (x - kS5R >= 0) && (x + kS5R <= W - 1) &&
                                      (x - kS5R - minD - d0 - 3 >= 0) && (d0 + 4 <= D);
                if (interior) {
                    outw = __umulhi(s0, mfull) | (__umulhi(s1, mfull) << 8) | (__umulhi(s2, mfull) << 16) |
                           (__umulhi(s3, mfull) << 24);
                } else {
                    const uint32_t sv[4] = {s0, s1, s2, s3};
                    outw = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int d = d0 + b;
                        uint32_t v;
                        if (d >= D) {
                            v = 0;
                        } else {
                            const int ad = minD + d;
                            const int clo = max(max(-kS5R, -x), ad - x);
                            const int chi = min(kS5R, W - 1 - x);
                            const int cnt = cy * max(0, chi - clo + 1);
                            v = cnt > 0 ? (cnt == 1 ? sv[b] : __umulhi(sv[b], magic[cnt])) : 255u;
                        }
                        outw |= v << (8 * b);
                    }
                }
                *reinterpret_cast<uint32_t*>(crow + (size_t)x * Dp) = outw;
            }
        }
        __syncthreads();
    }
}

// ceil(2^32 / c) for c >= 2 (c = 0, 1 unused): sum / c == umulhi(sum, m[c])
// whenever sum * (m[c]*c - 2^32) < 2^32, which holds for every SAD window sum.
__global__ void magic_kernel(uint32_t* m, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    m[c] = c >= 2 ? (uint32_t)((0x100000000ull + (unsigned long long)c - 1ull) /
                               (unsigned long long)c)
                  : 0u;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t launch_magic(uint32_t* m, int n, cudaStream_t s) {
    magic_kernel<<<(n + 255) / 256, 256, 0, s>>>(m, n);
    return cudaGetLastError();
}

void launch_stage_gray(const uint8_t* l, const uint8_t* r, size_t pitch, int channels, int W,
                       int H, uint8_t* gl, uint8_t* gr, cudaStream_t s, int nImages) {
    dim3 g((W + 255) / 256, H, nImages);
    stage_gray_kernel<<<g, 256, 0, s>>>(l, r, pitch, channels, W, H, gl, gr);
}

void launch_prefilter(const uint8_t* gl, const uint8_t* gr, int W, int H, int cap, uint8_t* pl,
                      uint8_t* pr, cudaStream_t s) {
    dim3 g((W + 255) / 256, H, 2);
    prefilter_kernel<<<g, 256, 0, s>>>(gl, gr, W, H, cap, pl, pr);
}

void launch_census(const uint8_t* gl, const uint8_t* gr, int W, int H, uint32_t* cl, uint32_t* cr,
                   cudaStream_t s) {
    dim3 g((W + 15) / 16, (H + 15) / 16, 2);
    census_kernel<<<g, dim3(16, 16), 0, s>>>(gl, gr, W, H, cl, cr);
}

cudaError_t launch_census_cost(const uint32_t* cl, const uint32_t* cr, int W, int H, int D,
                               int Dp, int minD, uint8_t* cost, cudaStream_t s) {
    const size_t smem = census_smem_bytes(Dp);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(census_cost_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 g((W + kCensusTile - 1) / kCensusTile, H);
    // one thread a (4-pixel group, 16-disparity chunk) item, up to 256
    const int threads = std::min(256, (kCensusTile / kCensusPx) * (Dp / 16));
    census_cost_kernel<<<g, threads, smem, s>>>(cl, cr, W, H, D, Dp, minD, cost);
    return cudaGetLastError();
}

template <bool WIDE>
static cudaError_t launch_sad_kp(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int Dp,
                                 int minD, int r, const uint32_t* magic, uint8_t* cost, size_t smem,
                                 cudaStream_t s) {
    dim3 g((W + kSadTile - 1) / kSadTile, (H + kSadBand - 1) / kSadBand);
#define LUMEN_SAD_CASE(KP)                                                                     \
    case KP: {                                                                                 \
        auto kern = sad_cost_kernel<WIDE, KP>;                                                 \
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                             (int)smem);                                       \
        if (e != cudaSuccess) return e;                                                        \
        kern<<<g, 256, smem, s>>>(pl, pr, W, H, D, minD, r, magic, cost);                       \
        return cudaGetLastError();                                                             \
    }
    switch (Dp / 64) {
        LUMEN_SAD_CASE(1)
        LUMEN_SAD_CASE(2)
        LUMEN_SAD_CASE(3)
        LUMEN_SAD_CASE(4)
        LUMEN_SAD_CASE(5)
        LUMEN_SAD_CASE(6)
        LUMEN_SAD_CASE(7)
        LUMEN_SAD_CASE(8)
    default: return cudaErrorInvalidValue;
    }
#undef LUMEN_SAD_CASE
}

size_t sad_cost_smem(int Dp, int r) {
    const SadGeom g = sad_geom(Dp, r);
    return (size_t)((g.ring * (g.ncolp + g.rw) + 15) & ~15) + (size_t)g.ncol * (Dp / 4) * 8;
}

template <int KP>
static cudaError_t launch_sad5(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int minD,
                               const uint32_t* magic, uint8_t* cost, cudaStream_t s) {
    dim3 g((W + kS5X - 1) / kS5X, (H + kS5Y - 1) / kS5Y);
    sad5_cost_kernel<KP><<<g, s5_quads(KP) * s5_cln(KP), 0, s>>>(pl, pr, W, H, D, minD, magic, cost);
    return cudaGetLastError();
}

cudaError_t launch_sad_cost(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int Dp,
                            int minD, int r, const uint32_t* magic, int wide, uint8_t* cost,
                            cudaStream_t s) {
    if (r == kS5R && !wide) {
        switch (Dp / 64) {
        case 1: return launch_sad5<1>(pl, pr, W, H, D, minD, magic, cost, s);
        case 2: return launch_sad5<2>(pl, pr, W, H, D, minD, magic, cost, s);
        case 3: return launch_sad5<3>(pl, pr, W, H, D, minD, magic, cost, s);
        case 4: return launch_sad5<4>(pl, pr, W, H, D, minD, magic, cost, s);
        case 5: return launch_sad5<5>(pl, pr, W, H, D, minD, magic, cost, s);
        case 6: return launch_sad5<6>(pl, pr, W, H, D, minD, magic, cost, s);
        case 7: return launch_sad5<7>(pl, pr, W, H, D, minD, magic, cost, s);
        default: break;  // Dp = 512: its column sums exceed the static shared memory
        }
    }
    const size_t smem = sad_cost_smem(Dp, r);
    return wide ? launch_sad_kp<true>(pl, pr, W, H, D, Dp, minD, r, magic, cost, smem, s)
                : launch_sad_kp<false>(pl, pr, W, H, D, Dp, minD, r, magic, cost, smem, s);
}

}  // namespace lumen
