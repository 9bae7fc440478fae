// cost.cu -- input staging, prefilter, census and the uint8 cost volumes.
//
// Volume layout: cost[(y*W + x)*Dp + d], d fastest, Dp = D rounded up to 64;
// entries d >= D are 0.  Values for d < D equal the reference's:
//   SAD    src/sgbm_kernels.cu:70-212   integer mean of |Lf-Rf| over the valid
//                                       part of the window, 255 if none valid
//   Census src/sgbm_kernels.cu:250-286  (h*255+12)/24, 255 in the 2-px border
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
// 64-pixel tile); the right descriptors the tile can reach are staged in
// shared memory; each thread writes 16 consecutive disparities of one pixel
// as one 16-byte store (a warp's stores are contiguous).  Interior pixels
// (every reachable right pixel inside the 2-px border) skip the per-disparity
// border tests and convert two Hamming distances per instruction:
// ((85*(h0 | h1<<16) + 0x40004) >> 3) & 0x00FF00FF.
constexpr int kCensusTile = 64;
__global__ void __launch_bounds__(256)
census_cost_kernel(const uint32_t* __restrict__ cl, const uint32_t* __restrict__ cr, int W,
                   int H, int D, int Dp, int minD, uint8_t* __restrict__ cost) {
    extern __shared__ uint32_t sm_cr[];  // kCensusTile + Dp - 1 entries
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * kCensusTile;
    const int lo = x0 - minD - (Dp - 1);  // leftmost right-image column reached
    const int n = kCensusTile + Dp - 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int rx = lo + i;
        sm_cr[i] = (rx >= 0 && rx < W) ? cr[(size_t)y * W + rx] : 0u;
    }
    __syncthreads();
    const int chunks = Dp / 16;
    const int items = kCensusTile * chunks;
    const bool rowOk = (y >= 2 && y < H - 2);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int px = it / chunks, ch = it - px * chunks;
        const int x = x0 + px;
        if (x >= W) continue;
        const bool leftOk = rowOk && x >= 2 && x < W - 2;
        const int dlo = ch * 16;
        const int rxHi = x - minD - dlo, rxLo = rxHi - 15;  // right columns of this chunk
        uint32_t wv[4];
        if (leftOk && rxLo >= 2 && rxHi < W - 2 && dlo + 16 <= D) {
            const uint32_t a = cl[(size_t)y * W + x];
            const uint32_t* rp = sm_cr + (rxHi - lo);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t h0 = __popc(a ^ rp[-(4 * q + 0)]);
                const uint32_t h1 = __popc(a ^ rp[-(4 * q + 1)]);
                const uint32_t h2 = __popc(a ^ rp[-(4 * q + 2)]);
                const uint32_t h3 = __popc(a ^ rp[-(4 * q + 3)]);
                const uint32_t c02 = ((85u * (h0 | (h2 << 16)) + 0x40004u) >> 3) & 0x00FF00FFu;
                const uint32_t c13 = ((85u * (h1 | (h3 << 16)) + 0x40004u) >> 3) & 0x00FF00FFu;
                wv[q] = c02 | (c13 << 8);
            }
        } else {
            const uint32_t a = leftOk ? cl[(size_t)y * W + x] : 0u;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t packed = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int d = dlo + q * 4 + b;
                    const int rx = x - minD - d;
                    uint32_t c;
                    if (d >= D) c = 0u;
                    else if (!leftOk || rx < 2 || rx >= W - 2) c = 255u;
                    else c = census_cost_of(__popc(a ^ sm_cr[rx - lo]));
                    packed |= c << (8 * b);
                }
                wv[q] = packed;
            }
        }
        *reinterpret_cast<uint4*>(cost + ((size_t)y * W + x) * Dp + dlo) =
            make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
}

// ---------------------------------------------------------------------------
// SAD cost (src/sgbm_kernels.cu:70-212).  One CTA per (row y, 64-pixel tile).
// Shared memory holds the prefiltered rows y-r..y+r of both images (right rows
// reversed, so that four consecutive disparities of one column are four
// consecutive bytes), then the column sums
//   cs[x'][d] = sum over valid rows of |Lf(x',row) - Rf(x'-ad,row)|
// (0 for a column whose left or right pixel lies outside the image), four
// disparities per __vabsdiffu4.  The window sum adds 2r+1 column sums; the
// count is (#valid rows) x (#valid columns) and sum/count is
// umulhi(sum, ceil(2^32/count)), exact because sum*count < 2^32 here.
// `wide` selects 32-bit window sums when (2r+1)^2 * 2*cap can exceed 65535.
// ---------------------------------------------------------------------------
constexpr int kSadTile = 64;

__device__ __forceinline__ uint32_t load_u32_unaligned(const uint8_t* base, int i) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(base + (i & ~3));
    return __byte_perm(w[0], w[1], (uint32_t)(0x3210 + 0x1111 * (i & 3)));
}

__global__ void __launch_bounds__(256)
sad_cost_kernel(const uint8_t* __restrict__ pl, const uint8_t* __restrict__ pr, int W, int H,
                int D, int Dp, int minD, int r, const uint32_t* __restrict__ magic, int wide,
                uint8_t* __restrict__ cost) {
    extern __shared__ __align__(16) uint8_t sm[];
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * kSadTile;
    const int nrow = 2 * r + 1;
    const int ncol = kSadTile + 2 * r;             // columns x' of the column sums
    const int lx0 = x0 - r;                        // first column x'
    // Right row span, stored reversed: index j holds Rf(rtop - j).
    const int rtop = lx0 + ncol - 1 - minD;        // rightmost right column reached
    const int rw = (ncol + Dp - 1 + 3 + 4) & ~3;   // padded span (+4 slack for unaligned reads)
    uint8_t* sL = sm;                              // [nrow][ncolp]
    const int ncolp = (ncol + 3) & ~3;
    uint8_t* sR = sL + nrow * ncolp;               // [nrow][rw]
    uint32_t* cs = reinterpret_cast<uint32_t*>(
        sm + ((nrow * (ncolp + rw) + 15) & ~15));  // [ncol][Dp/2] packed pairs
    const int ylo = max(0, y - r), yhi = min(H - 1, y + r);
    const int cy = yhi - ylo + 1;
    for (int i = threadIdx.x; i < nrow * ncolp; i += blockDim.x) {
        const int rr = i / ncolp, c = i - rr * ncolp;
        const int gy = y - r + rr, gx = lx0 + c;
        sL[i] = (gy >= 0 && gy < H && gx >= 0 && gx < W && c < ncol) ? pl[(size_t)gy * W + gx] : 0;
    }
    for (int i = threadIdx.x; i < nrow * rw; i += blockDim.x) {
        const int rr = i / rw, j = i - rr * rw;
        const int gy = y - r + rr, gx = rtop - j;
        sR[i] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? pr[(size_t)gy * W + gx] : 0;
    }
    __syncthreads();
    // Column sums: 4 disparities per item.
    const int quads = Dp / 4;
    for (int it = threadIdx.x; it < ncol * quads; it += blockDim.x) {
        const int c = it / quads, q = it - c * quads;
        const int xg = lx0 + c;
        const int d0 = 4 * q;
        // byte b of the quad is disparity d0+b: right column xg - minD - d0 - b,
        // reversed index j = rtop - (xg - minD - d0 - b) = j0 + b.
        const int j0 = rtop - (xg - minD - d0);
        uint32_t mask = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int rx = xg - minD - d0 - b;
            if (xg >= 0 && xg < W && rx >= 0 && rx < W && d0 + b < D) mask |= 0xFFu << (8 * b);
        }
        uint32_t ev = 0, od = 0;  // (d0, d0+2) and (d0+1, d0+3) as u16 pairs
        if (mask) {
            for (int gy = ylo; gy <= yhi; ++gy) {
                const int rr = gy - (y - r);
                const uint32_t l4 = (uint32_t)sL[rr * ncolp + c] * 0x01010101u;
                const uint32_t r4 = load_u32_unaligned(sR + rr * rw, j0);
                const uint32_t v = __vabsdiffu4(l4, r4) & mask;
                ev += v & 0x00FF00FFu;
                od += (v >> 8) & 0x00FF00FFu;
            }
        }
        cs[c * (Dp / 2) + 2 * q] = __byte_perm(ev, od, 0x5410);
        cs[c * (Dp / 2) + 2 * q + 1] = __byte_perm(ev, od, 0x7632);
    }
    __syncthreads();
    // Window sums, 16 disparities per item (one 16-byte store).
    const int chunks = Dp / 16;
    for (int it = threadIdx.x; it < kSadTile * chunks; it += blockDim.x) {
        const int px = it / chunks, ch = it - px * chunks;
        const int x = x0 + px;
        if (x >= W) continue;
        uint32_t s[16];
        if (!wide) {
            uint32_t sums[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) sums[k] = 0;
            for (int dx = -r; dx <= r; ++dx) {
                const uint4* src = reinterpret_cast<const uint4*>(cs + (size_t)(px + r + dx) * (Dp / 2) + ch * 8);
                const uint4 a = src[0], b = src[1];
                sums[0] += a.x; sums[1] += a.y; sums[2] += a.z; sums[3] += a.w;
                sums[4] += b.x; sums[5] += b.y; sums[6] += b.z; sums[7] += b.w;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) { s[2 * k] = sums[k] & 0xFFFFu; s[2 * k + 1] = sums[k] >> 16; }
        } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) s[k] = 0;
            for (int dx = -r; dx <= r; ++dx) {
                const uint32_t* src = cs + (size_t)(px + r + dx) * (Dp / 2) + ch * 8;
#pragma unroll
                for (int k = 0; k < 8; ++k) { s[2 * k] += src[k] & 0xFFFFu; s[2 * k + 1] += src[k] >> 16; }
            }
        }
        const int dlo = ch * 16;
        uint32_t outw[4];
        const int full = (2 * r + 1) * cy;
        const bool interior = (x - r >= 0) && (x + r <= W - 1) && (x - r - minD - (dlo + 15) >= 0) &&
                              (x + r - minD - dlo <= W - 1) && (dlo + 16 <= D);
        if (interior) {
            const uint32_t m = magic[full];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t packed = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    packed |= (full == 1 ? s[4 * q + b] : __umulhi(s[4 * q + b], m)) << (8 * b);
                outw[q] = packed;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t packed = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int d = dlo + 4 * q + b;
                    uint32_t v;
                    if (d >= D) {
                        v = 0;
                    } else {
                        // valid columns: x+dx in [0,W) and x+dx-ad in [0,W)
                        const int ad = minD + d;
                        const int clo = max(max(-r, -x), ad - x);
                        const int chi = min(min(r, W - 1 - x), W - 1 - x + ad);
                        const int cnt = cy * max(0, chi - clo + 1);
                        v = cnt > 0 ? (cnt == 1 ? s[4 * q + b] : __umulhi(s[4 * q + b], magic[cnt])) : 255u;
                    }
                    packed |= v << (8 * b);
                }
                outw[q] = packed;
            }
        }
        *reinterpret_cast<uint4*>(cost + ((size_t)y * W + x) * Dp + dlo) =
            make_uint4(outw[0], outw[1], outw[2], outw[3]);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
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
    const size_t smem = (size_t)(kCensusTile + Dp - 1) * 4;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(census_cost_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 g((W + kCensusTile - 1) / kCensusTile, H);
    census_cost_kernel<<<g, 256, smem, s>>>(cl, cr, W, H, D, Dp, minD, cost);
    return cudaGetLastError();
}

size_t sad_cost_smem(int Dp, int r) {
    const int nrow = 2 * r + 1, ncol = kSadTile + 2 * r;
    const int ncolp = (ncol + 3) & ~3, rw = (ncol + Dp - 1 + 3 + 4) & ~3;
    return (size_t)((nrow * (ncolp + rw) + 15) & ~15) + (size_t)ncol * Dp * 2;
}

cudaError_t launch_sad_cost(const uint8_t* pl, const uint8_t* pr, int W, int H, int D, int Dp,
                            int minD, int r, const uint32_t* magic, int wide, uint8_t* cost,
                            cudaStream_t s) {
    const size_t smem = sad_cost_smem(Dp, r);
    cudaError_t e = cudaFuncSetAttribute(sad_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 g((W + kSadTile - 1) / kSadTile, H);
    sad_cost_kernel<<<g, 256, smem, s>>>(pl, pr, W, H, D, Dp, minD, r, magic, wide, cost);
    return cudaGetLastError();
}

}  // namespace lumen
