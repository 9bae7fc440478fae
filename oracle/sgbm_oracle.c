/*
 * sgbm_oracle.c -- CPU restatement of LumenStereo's SGBM stereo path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * lumenstereo_b200/ and the timed CPU baseline in bench.py; nothing in the
 * product links it, calls it or falls back to it.  Every function restates one
 * reference kernel (or host step) and cites the file:line it follows, paths
 * relative to the LumenStereo source tree.  Integer stages are restated with
 * the exact C integer semantics the reference's CUDA code has (uint16 wrap on
 * every assignment, int promotion inside expressions, truncating division).
 * The one floating-point stage (parabola subpixel) uses IEEE single precision
 * here; the reference is compiled with --use_fast_math, so its division may
 * differ by an ulp (see the subpixel tolerance in the tests).
 *
 * Parallelism: OpenMP over independent rows / path lines when built with
 * -fopenmp (used for the CPU baseline); results do not depend on the thread
 * count (every parallel loop writes disjoint outputs, paths are accumulated in
 * a fixed order).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Same field order as lumen_stereo_params in include/lumen_sgbm.h and
 * stereo::StereoParams (include/stereo/stereo_params.h:57-82 in the reference). */
typedef struct oracle_params {
    int minDisparity;
    int maxDisparity;
    int blockSize;
    int P1;
    int P2;
    int preFilterCap;
    int uniquenessRatio;
    int disp12MaxDiff;
    int speckleWindowSize;
    int speckleRange;
    int useGPU;
    int useSharedMemory;
    int numDirections;
    int matchingCostMode; /* 0 = SAD, 1 = Census */
} oracle_params;

/* Optional intermediate outputs of oracle_sgbm_compute (any may be NULL). */
typedef struct oracle_intermediates {
    uint8_t* gray_left;     /* W*H */
    uint8_t* gray_right;    /* W*H */
    uint8_t* pref_left;     /* W*H, SAD mode */
    uint8_t* pref_right;    /* W*H, SAD mode */
    uint32_t* census_left;  /* W*H, Census mode */
    uint32_t* census_right; /* W*H, Census mode */
    uint8_t* cost;          /* W*H*D */
    uint16_t* agg;          /* W*H*D */
    int16_t* disp_wta;      /* W*H, left WTA before LR */
    int16_t* disp_right;    /* W*H */
    int16_t* disp_lr;       /* W*H, after LR check (and speckle when enabled) */
} oracle_intermediates;

#define ORACLE_MAX_DISPARITY_RANGE 512 /* include/stereo/sgbm_limits.h:9 */

enum {
    ORACLE_OK = 0,
    ORACLE_ERR_INVALID_ARGUMENT = 1,
    ORACLE_ERR_RANGE_EXCEEDS_LIMIT = 2,
    ORACLE_ERR_OUT_OF_MEMORY = 4
};

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* src/sgbm_kernels.cu:38-59 (prefilterXSobel): one-row central difference,
 * one-sided at x = 0 and x = W-1, clipped to [-cap, cap], shifted by +cap. */
void oracle_prefilter_xsobel(const uint8_t* img, uint8_t* out, int W, int H, int cap) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        const uint8_t* row = img + (size_t)y * W;
        for (int x = 0; x < W; ++x) {
            int val;
            if (x > 0 && x < W - 1) val = (int)row[x + 1] - (int)row[x - 1];
            else if (x == 0) val = (int)row[1] - (int)row[0];
            else val = (int)row[x] - (int)row[x - 1];
            val = imin(cap, imax(-cap, val));
            out[(size_t)y * W + x] = (uint8_t)(val + cap);
        }
    }
}

/* src/sgbm_kernels.cu:217-245 (buildCensus5x5): 24-bit descriptor, row-major
 * over the 5x5 window minus the centre, bit set when neighbour >= centre;
 * 2-pixel border -> 0. */
void oracle_census5x5(const uint8_t* img, uint32_t* census, int W, int H) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            if (x < 2 || x >= W - 2 || y < 2 || y >= H - 2) {
                census[(size_t)y * W + x] = 0u;
                continue;
            }
            const uint8_t c = img[(size_t)y * W + x];
            uint32_t bits = 0u;
            int bit = 0;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    if (img[(size_t)(y + dy) * W + (x + dx)] >= c) bits |= (1u << bit);
                    ++bit;
                }
            census[(size_t)y * W + x] = bits;
        }
    }
}

/* src/sgbm_kernels.cu:172-212 (computeCostSAD_naive; the shared-memory
 * variant at :70-167 computes the same values): integer mean of |Lf - Rf| over
 * the valid part of the (2r+1)^2 window, 255 when nothing is valid. */
void oracle_cost_sad(const uint8_t* lf, const uint8_t* rf, uint8_t* cost, int W, int H,
                     int D, int minD, int radius) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            uint8_t* out = cost + ((size_t)y * W + x) * (size_t)D;
            for (int d = 0; d < D; ++d) {
                const int ad = minD + d;
                int sum = 0, count = 0;
                for (int dy = -radius; dy <= radius; ++dy) {
                    const int ly = y + dy;
                    if (ly < 0 || ly >= H) continue;
                    const uint8_t* lrow = lf + (size_t)ly * W;
                    const uint8_t* rrow = rf + (size_t)ly * W;
                    for (int dx = -radius; dx <= radius; ++dx) {
                        const int lx = x + dx;
                        const int rx = lx - ad;
                        if (lx >= 0 && lx < W && rx >= 0 && rx < W) {
                            sum += abs((int)lrow[lx] - (int)rrow[rx]);
                            ++count;
                        }
                    }
                }
                out[d] = (uint8_t)(count > 0 ? sum / count : 255);
            }
        }
    }
}

/* src/sgbm_kernels.cu:250-286 (computeCostCensus_naive): Hamming distance of
 * the descriptors scaled to 0..255 as (h*255+12)/24; 255 when the left pixel
 * or the matched right pixel lies in the 2-pixel border. */
void oracle_cost_census(const uint32_t* cl, const uint32_t* cr, uint8_t* cost, int W, int H,
                        int D, int minD) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            uint8_t* out = cost + ((size_t)y * W + x) * (size_t)D;
            const int leftOk = (x >= 2 && x < W - 2 && y >= 2 && y < H - 2);
            if (!leftOk) {
                memset(out, 255, (size_t)D);
                continue;
            }
            const uint32_t a = cl[(size_t)y * W + x];
            for (int d = 0; d < D; ++d) {
                const int rx = x - (minD + d);
                if (!(rx >= 2 && rx < W - 2)) {
                    out[d] = 255;
                    continue;
                }
                const int h = __builtin_popcount(a ^ cr[(size_t)y * W + rx]);
                out[d] = (uint8_t)((h * 255 + 12) / 24);
            }
        }
    }
}

/* src/sgbm_kernels.cu:304-310 (adaptiveP2). */
static inline int adaptive_p2(int P1, int P2, int cur, int prev) {
    const int g = abs(cur - prev);
    return imax(P1 + 1, P2 * 8 / imax(8, g));
}

/* One SGM path line: src/sgbm_kernels.cu:315-361 (and the seven sibling
 * kernels up to :742 differ only in the walk).  The first pixel of the line
 * takes L = C (:333-336, :541-546); every later pixel applies
 *   L[d] = (u16)(C + min(L'[d], (u16)(L'[d-1]+P1), (u16)(L'[d+1]+P1),
 *                        (u16)(minL' + P2adj)) - minL')
 * with out-of-range neighbours = 0xFFFF, and agg[p][d] += L[d] (mod 2^16). */
static void sgm_line(const uint8_t* cost, const uint8_t* img, uint16_t* agg, int W, int D,
                     int P1, int P2, int costScale, int x, int y, int sx, int sy, int H,
                     uint16_t* Lp, uint16_t* Lc) {
    size_t p = (size_t)y * W + x;
    for (int d = 0; d < D; ++d) {
        Lp[d] = (uint16_t)((int)cost[p * D + d] * costScale);
        agg[p * D + d] = (uint16_t)(agg[p * D + d] + Lp[d]);
    }
    int px = x, py = y;
    x += sx;
    y += sy;
    while (x >= 0 && x < W && y >= 0 && y < H) {
        p = (size_t)y * W + x;
        const int P2adj = adaptive_p2(P1, P2, img[p], img[(size_t)py * W + px]);
        uint16_t minPrev = 0xFFFF;
        for (int d = 0; d < D; ++d)
            if (Lp[d] < minPrev) minPrev = Lp[d];
        for (int d = 0; d < D; ++d) {
            const uint16_t C = (uint16_t)((int)cost[p * D + d] * costScale);
            const uint16_t c0 = Lp[d];
            const uint16_t c1 = (d > 0) ? (uint16_t)(Lp[d - 1] + P1) : (uint16_t)0xFFFF;
            const uint16_t c2 = (d < D - 1) ? (uint16_t)(Lp[d + 1] + P1) : (uint16_t)0xFFFF;
            const uint16_t c3 = (uint16_t)(minPrev + P2adj);
            uint16_t m = c0 < c1 ? c0 : c1;
            const uint16_t m2 = c2 < c3 ? c2 : c3;
            m = m < m2 ? m : m2;
            Lc[d] = (uint16_t)(C + m - minPrev);
            agg[p * D + d] = (uint16_t)(agg[p * D + d] + Lc[d]);
        }
        uint16_t* t = Lp;
        Lp = Lc;
        Lc = t;
        px = x;
        py = y;
        x += sx;
        y += sy;
    }
}

/* Path bit order (same as the launch order in src/sgbm_gpu.cu:321-421). */
enum {
    PATH_LR = 1u << 0,
    PATH_RL = 1u << 1,
    PATH_TB = 1u << 2,
    PATH_BT = 1u << 3,
    PATH_TLBR = 1u << 4,
    PATH_BRTL = 1u << 5,
    PATH_TRBL = 1u << 6,
    PATH_BLTR = 1u << 7
};

/* Start pixels of every line of one direction, in the same order for every
 * call.  Returns the number of lines; (xs[i], ys[i]) is the first pixel. */
static int path_starts(int dir, int W, int H, int* xs, int* ys, int* sx, int* sy) {
    int n = 0;
    switch (dir) {
    case 0: *sx = 1; *sy = 0;  for (int y = 0; y < H; ++y) { xs[n] = 0; ys[n++] = y; } break;
    case 1: *sx = -1; *sy = 0; for (int y = 0; y < H; ++y) { xs[n] = W - 1; ys[n++] = y; } break;
    case 2: *sx = 0; *sy = 1;  for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = 0; } break;
    case 3: *sx = 0; *sy = -1; for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = H - 1; } break;
    case 4: /* TLBR, :519-571: start where x == 0 || y == 0 */
        *sx = 1; *sy = 1;
        for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = 0; }
        for (int y = 1; y < H; ++y) { xs[n] = 0; ys[n++] = y; }
        break;
    case 5: /* BRTL, :576-628: start where x == W-1 || y == H-1 */
        *sx = -1; *sy = -1;
        for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = H - 1; }
        for (int y = 0; y < H - 1; ++y) { xs[n] = W - 1; ys[n++] = y; }
        break;
    case 6: /* TRBL, :633-685: start where x == W-1 || y == 0 */
        *sx = -1; *sy = 1;
        for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = 0; }
        for (int y = 1; y < H; ++y) { xs[n] = W - 1; ys[n++] = y; }
        break;
    default: /* BLTR, :690-742: start where x == 0 || y == H-1 */
        *sx = 1; *sy = -1;
        for (int x = 0; x < W; ++x) { xs[n] = x; ys[n++] = H - 1; }
        for (int y = 0; y < H - 1; ++y) { xs[n] = 0; ys[n++] = y; }
        break;
    }
    return n;
}

/* src/sgbm_gpu.cu:297-430 (aggregateCosts): agg = 0, then every selected path
 * adds its L into agg.  pathMask selects paths by the PATH_* bits (the
 * reference runs LR, RL, TB, BT always and the four diagonals when
 * numDirections >= 8).  Returns nonzero on allocation failure. */
int oracle_aggregate(const uint8_t* cost, const uint8_t* img, uint16_t* agg, int W, int H, int D,
                     int P1, int P2, int costScale, unsigned pathMask) {
    memset(agg, 0, (size_t)W * H * D * sizeof(uint16_t));
    int* xs = (int*)malloc(sizeof(int) * (size_t)(W + H));
    int* ys = (int*)malloc(sizeof(int) * (size_t)(W + H));
    if (!xs || !ys) { free(xs); free(ys); return ORACLE_ERR_OUT_OF_MEMORY; }
    int rc = ORACLE_OK;
    for (int dir = 0; dir < 8; ++dir) {
        if (!(pathMask & (1u << dir))) continue;
        int sx, sy;
        const int n = path_starts(dir, W, H, xs, ys, &sx, &sy);
        /* Lines of one direction touch disjoint pixels: parallel and race-free. */
        #pragma omp parallel
        {
            uint16_t* buf = (uint16_t*)malloc(sizeof(uint16_t) * 2 * (size_t)D);
            if (!buf) {
                #pragma omp atomic write
                rc = ORACLE_ERR_OUT_OF_MEMORY;
            } else {
                #pragma omp for schedule(dynamic, 16)
                for (int i = 0; i < n; ++i)
                    sgm_line(cost, img, agg, W, D, P1, P2, costScale, xs[i], ys[i], sx, sy, H, buf,
                             buf + D);
                free(buf);
            }
        }
    }
    free(xs);
    free(ys);
    return rc;
}

/* Parabola subpixel of src/sgbm_kernels.cu:789-804 (and :836-855). */
static inline int16_t subpixel_out(const uint16_t* v, int bestD, int D, int minD) {
    float subpixelD = (float)bestD;
    if (bestD > 0 && bestD < D - 1) {
        const float c0 = (float)v[bestD - 1];
        const float c1 = (float)v[bestD];
        const float c2 = (float)v[bestD + 1];
        const float denom = 2.0f * (c0 + c2 - 2.0f * c1);
        if (fabsf(denom) > 1e-6f) {
            float delta = (c0 - c2) / denom;
            delta = fmaxf(-1.0f, fminf(1.0f, delta));
            subpixelD += delta;
        }
    }
    return (int16_t)(int)((subpixelD + (float)minD) * 16.0f);
}

/* src/sgbm_kernels.cu:748-805 (selectDisparityWTA): first strict minimum,
 * running second minimum, uniqueness test, parabola subpixel, 1/16 px. */
void oracle_select_wta(const uint16_t* agg, int16_t* disp, int W, int H, int D, int minD, int UR) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const uint16_t* v = agg + ((size_t)y * W + x) * (size_t)D;
            uint16_t minCost = 0xFFFF, second = 0xFFFF;
            int bestD = 0;
            for (int d = 0; d < D; ++d) {
                const uint16_t c = v[d];
                if (c < minCost) { second = minCost; minCost = c; bestD = d; }
                else if (c < second) second = c;
            }
            if (UR > 0 && second != 0xFFFF) {
                const uint32_t best = minCost;
                const uint32_t thresh = (best * (uint32_t)UR) / 100u;
                if ((uint32_t)second <= best + thresh) {
                    disp[(size_t)y * W + x] = -1;
                    continue;
                }
            }
            disp[(size_t)y * W + x] = subpixel_out(v, bestD, D, minD);
        }
    }
}

/* src/sgbm_kernels.cu:807-856 (selectDisparityRight): right-view argmin over
 * agg[y][x+minD+d][d], stopping at the image edge; subpixel from the left
 * pixel's d-1, d, d+1 (the reference's choice, kept). */
void oracle_select_right(const uint16_t* agg, int16_t* dispR, int W, int H, int D, int minD) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            uint16_t minCost = 0xFFFF;
            int bestD = 0;
            for (int d = 0; d < D; ++d) {
                const int lx = x + minD + d;
                if (lx >= W) break;
                const uint16_t c = agg[((size_t)y * W + lx) * (size_t)D + d];
                if (c < minCost) { minCost = c; bestD = d; }
            }
            int16_t out;
            const int lx = x + minD + bestD;
            if (bestD > 0 && bestD < D - 1 && lx < W)
                out = subpixel_out(agg + ((size_t)y * W + lx) * (size_t)D, bestD, D, minD);
            else
                out = (int16_t)(int)(((float)bestD + (float)minD) * 16.0f);
            dispR[(size_t)y * W + x] = out;
        }
    }
}

/* src/sgbm_kernels.cu:862-890 (consistencyCheck), in place. */
void oracle_consistency(int16_t* dispL, const int16_t* dispR, int W, int H, int maxDiff) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const int16_t dL = dispL[(size_t)y * W + x];
            if (dL <= 0) continue;
            const int xR = x - dL / 16;
            if (xR < 0 || xR >= W) { dispL[(size_t)y * W + x] = -1; continue; }
            const int16_t dR = dispR[(size_t)y * W + xR];
            if (dR <= 0 || abs((int)dL - (int)dR) > maxDiff) dispL[(size_t)y * W + x] = -1;
        }
    }
}

/* src/sgbm_kernels.cu:979-1013 (speckleFilter) with read-from-snapshot
 * semantics.  The reference kernel reads neighbours in place while other
 * threads write -1 (a data race, so its output depends on scheduling); this
 * restatement reads the pre-filter map, which is the deterministic meaning. */
void oracle_speckle(int16_t* disp, int W, int H, int maxSpeckleSize, int maxDiff) {
    const size_t n = (size_t)W * H;
    int16_t* snap = (int16_t*)malloc(n * sizeof(int16_t));
    if (!snap) return;
    memcpy(snap, disp, n * sizeof(int16_t));
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const int16_t c = snap[(size_t)y * W + x];
            if (c <= 0) continue;
            int similar = 0;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    const int nx = x + dx, ny = y + dy;
                    if (nx >= 0 && nx < W && ny >= 0 && ny < H) {
                        const int16_t v = snap[(size_t)ny * W + nx];
                        if (v > 0 && abs((int)c - (int)v) <= maxDiff) ++similar;
                    }
                }
            if (similar < maxSpeckleSize) disp[(size_t)y * W + x] = -1;
        }
    }
    free(snap);
}

/* src/sgbm_kernels.cu:892-935 (medianFilter3x3): upper median of the positive
 * values in the 3x3 neighbourhood (centre included); copy when none. */
void oracle_median3x3(const int16_t* in, int16_t* out, int W, int H) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            int16_t v[9];
            int count = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = x + dx, ny = y + dy;
                    if (nx >= 0 && nx < W && ny >= 0 && ny < H) {
                        const int16_t val = in[(size_t)ny * W + nx];
                        if (val > 0) {
                            int j = count++;
                            while (j > 0 && v[j - 1] > val) { v[j] = v[j - 1]; --j; }
                            v[j] = val;
                        }
                    }
                }
            out[(size_t)y * W + x] = count == 0 ? in[(size_t)y * W + x] : v[count / 2];
        }
    }
}

/* src/rectification.cu:201-253 (remapKernelSimple): bilinear with floorf,
 * out-of-image taps read as 0, result truncated after +0.5.  The four-term
 * sum is evaluated as the chain of fused multiply-adds
 *   fma(w11,v11, fma(w10,v10, fma(w01,v01, w00*v00)))
 * which is the contraction of the left-to-right sum the CUDA compiler forms;
 * the tests check this against the reference kernel run on the GPU. */
void oracle_remap(const uint8_t* src, const float* mapX, const float* mapY, uint8_t* dst, int W,
                  int H, int channels) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t idx = (size_t)y * W + x;
            const float sxf = mapX[idx], syf = mapY[idx];
            const int x0 = (int)floorf(sxf), y0 = (int)floorf(syf);
            const int x1 = x0 + 1, y1 = y0 + 1;
            const float dx = sxf - (float)x0, dy = syf - (float)y0;
            const float w00 = (1.0f - dx) * (1.0f - dy);
            const float w01 = (1.0f - dx) * dy;
            const float w10 = dx * (1.0f - dy);
            const float w11 = dx * dy;
            const size_t rs = (size_t)W * channels;
            const int v00ok = x0 >= 0 && x0 < W && y0 >= 0 && y0 < H;
            const int v01ok = x0 >= 0 && x0 < W && y1 >= 0 && y1 < H;
            const int v10ok = x1 >= 0 && x1 < W && y0 >= 0 && y0 < H;
            const int v11ok = x1 >= 0 && x1 < W && y1 >= 0 && y1 < H;
            for (int c = 0; c < channels; ++c) {
                const float v00 = v00ok ? (float)src[(size_t)y0 * rs + (size_t)x0 * channels + c] : 0.0f;
                const float v01 = v01ok ? (float)src[(size_t)y1 * rs + (size_t)x0 * channels + c] : 0.0f;
                const float v10 = v10ok ? (float)src[(size_t)y0 * rs + (size_t)x1 * channels + c] : 0.0f;
                const float v11 = v11ok ? (float)src[(size_t)y1 * rs + (size_t)x1 * channels + c] : 0.0f;
                const float val = fmaf(w11, v11, fmaf(w10, v10, fmaf(w01, v01, w00 * v00)));
                dst[(size_t)y * rs + (size_t)x * channels + c] = (uint8_t)(int)(val + 0.5f);
            }
        }
    }
}

/* OpenCV cvtColor(COLOR_BGR2GRAY) for 8-bit input, which the reference calls
 * at src/sgbm_gpu.cu:169-172.  OpenCV 4.x computes BT.601 luma in 15-bit fixed
 * point with coefficients summing to 2^15:
 *   Y = (3735*B + 19235*G + 9798*R + 16384) >> 15
 * (OpenCV is an unpinned apt dependency of the reference; this formula equals
 * cv2 4.13's output on all 2^24 colours, checked in tests/test_oracle.py). */
void oracle_bgr2gray(const uint8_t* bgr, uint8_t* gray, int W, int H, size_t strideBytes) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        const uint8_t* row = bgr + (size_t)y * strideBytes;
        for (int x = 0; x < W; ++x) {
            const int b = row[3 * x], g = row[3 * x + 1], r = row[3 * x + 2];
            gray[(size_t)y * W + x] = (uint8_t)((3735 * b + 19235 * g + 9798 * r + 16384) >> 15);
        }
    }
}

/* costScale of src/sgbm_gpu.cu:312-317. */
int oracle_cost_scale(const oracle_params* p) {
    if (p->matchingCostMode == 0) return p->blockSize * p->blockSize;
    return imax(1, (p->blockSize * p->blockSize * 2 * p->preFilterCap) / 255);
}

unsigned oracle_path_mask(const oracle_params* p) {
    return p->numDirections >= 8 ? 0xFFu : (PATH_LR | PATH_RL | PATH_TB | PATH_BT);
}

/* src/sgbm_gpu.cu:147-195 and :197-515 (StereoSGBM::compute and its stages).
 * left/right: W*H*channels bytes, rows contiguous; disp: W*H int16 (1/16 px,
 * -1 = invalid).  pathMaskOverride != 0 replaces the path set (debug: one
 * path at a time). */
int oracle_sgbm_compute(const oracle_params* p, const uint8_t* left, const uint8_t* right, int W,
                        int H, int channels, int16_t* disp, oracle_intermediates* dbg,
                        unsigned pathMaskOverride) {
    if (!left || !right || W <= 0 || H <= 0) return ORACLE_ERR_INVALID_ARGUMENT; /* :148-150 */
    const int D = p->maxDisparity - p->minDisparity;
    if (D < 1) return ORACLE_ERR_INVALID_ARGUMENT;                               /* :159-161 */
    if (D > ORACLE_MAX_DISPARITY_RANGE) return ORACLE_ERR_RANGE_EXCEEDS_LIMIT;   /* :162-166 */
    if (channels != 1 && channels != 3) return ORACLE_ERR_INVALID_ARGUMENT;

    const size_t N = (size_t)W * H;
    const size_t ND = N * (size_t)D;
    uint8_t* gl = dbg && dbg->gray_left ? dbg->gray_left : (uint8_t*)malloc(N);
    uint8_t* gr = dbg && dbg->gray_right ? dbg->gray_right : (uint8_t*)malloc(N);
    uint8_t* cost = dbg && dbg->cost ? dbg->cost : (uint8_t*)malloc(ND);
    uint16_t* agg = dbg && dbg->agg ? dbg->agg : (uint16_t*)malloc(ND * sizeof(uint16_t));
    int16_t* dl = (int16_t*)malloc(N * sizeof(int16_t));
    int16_t* dr = (int16_t*)malloc(N * sizeof(int16_t));
    uint8_t* pl = NULL; uint8_t* pr = NULL; uint32_t* cl = NULL; uint32_t* cr = NULL;
    int rc = ORACLE_OK;
    if (!gl || !gr || !cost || !agg || !dl || !dr) { rc = ORACLE_ERR_OUT_OF_MEMORY; goto done; }

    if (channels == 3) { /* :169-172 */
        oracle_bgr2gray(left, gl, W, H, (size_t)W * 3);
        oracle_bgr2gray(right, gr, W, H, (size_t)W * 3);
    } else {
        memcpy(gl, left, N);
        memcpy(gr, right, N);
    }

    if (p->matchingCostMode == 1) { /* :206-222 */
        cl = dbg && dbg->census_left ? dbg->census_left : (uint32_t*)malloc(N * 4);
        cr = dbg && dbg->census_right ? dbg->census_right : (uint32_t*)malloc(N * 4);
        if (!cl || !cr) { rc = ORACLE_ERR_OUT_OF_MEMORY; goto done; }
        oracle_census5x5(gl, cl, W, H);
        oracle_census5x5(gr, cr, W, H);
        oracle_cost_census(cl, cr, cost, W, H, D, p->minDisparity);
    } else { /* :223-286 */
        const int cap = imax(1, p->preFilterCap);
        pl = dbg && dbg->pref_left ? dbg->pref_left : (uint8_t*)malloc(N);
        pr = dbg && dbg->pref_right ? dbg->pref_right : (uint8_t*)malloc(N);
        if (!pl || !pr) { rc = ORACLE_ERR_OUT_OF_MEMORY; goto done; }
        oracle_prefilter_xsobel(gl, pl, W, H, cap);
        oracle_prefilter_xsobel(gr, pr, W, H, cap);
        oracle_cost_sad(pl, pr, cost, W, H, D, p->minDisparity, p->blockSize / 2);
    }

    rc = oracle_aggregate(cost, gl, agg, W, H, D, p->P1, p->P2, oracle_cost_scale(p),
                          pathMaskOverride ? pathMaskOverride : oracle_path_mask(p));
    if (rc) goto done;

    oracle_select_wta(agg, dl, W, H, D, p->minDisparity, p->uniquenessRatio); /* :438-446 */
    oracle_select_right(agg, dr, W, H, D, p->minDisparity);                   /* :449-456 */
    if (dbg && dbg->disp_wta) memcpy(dbg->disp_wta, dl, N * sizeof(int16_t));
    if (dbg && dbg->disp_right) memcpy(dbg->disp_right, dr, N * sizeof(int16_t));
    if (p->disp12MaxDiff >= 0) oracle_consistency(dl, dr, W, H, p->disp12MaxDiff * 16); /* :469-478 */
    if (p->speckleWindowSize > 0)                                                       /* :480-490 */
        oracle_speckle(dl, W, H, imin(p->speckleWindowSize, 25), p->speckleRange * 16);
    if (dbg && dbg->disp_lr) memcpy(dbg->disp_lr, dl, N * sizeof(int16_t));
    oracle_median3x3(dl, disp, W, H); /* :493-507 */

done:
    if (!(dbg && dbg->gray_left)) free(gl);
    if (!(dbg && dbg->gray_right)) free(gr);
    if (!(dbg && dbg->cost)) free(cost);
    if (!(dbg && dbg->agg)) free(agg);
    if (!(dbg && dbg->pref_left)) free(pl);
    if (!(dbg && dbg->pref_right)) free(pr);
    if (!(dbg && dbg->census_left)) free(cl);
    if (!(dbg && dbg->census_right)) free(cr);
    free(dl);
    free(dr);
    return rc;
}
