// pair_layout.h -- the index arithmetic of schedule 6 (pair_kernel.cuh) that
// host and device share: sweep geometry, ticket order, band-boundary row
// buffers and the shared-memory carve-up.  Plain C++ so host tests compile it
// without nvcc (tests/cpp/pair_layout_test.cpp).
#pragma once
#include <cstddef>

#ifdef __CUDACC__
#define LUMEN_PAIR_HD __host__ __device__ __forceinline__
#else
#define LUMEN_PAIR_HD inline
#endif

namespace lumen {

constexpr int kPPF = 8;    // per-row cost ring (pixels); kPPF-1 prefetched ahead
constexpr int kPQ = 32;    // import ring: pixels of the band above held for row 0
constexpr int kPG = 8;     // pixels the import warp polls and copies at a time

// Shared-memory slot of one pixel's diagonal vector: Dp uint16 values, the
// vector's minimum (uint32) and padding to 16 bytes.
LUMEN_PAIR_HD constexpr int pair_slot_bytes(int Dp) { return 2 * Dp + 16; }

// Band-boundary row buffers hold, per pixel, the slot's Dp / 2 + 1 payload
// words as 64-bit (payload, epoch) words -- the epoch of the launch that wrote
// them in the high half -- padded to an even count so every pixel starts on a
// 16-byte boundary.  A reader takes a word once its epoch is the current one:
// no fence or progress counter is needed between the bands.
LUMEN_PAIR_HD constexpr int pair_ll_words(int Dp) { return Dp / 2 + 2; }

struct PairSmem {
    int img, cost, slots, imp, zero, lut, job, misc, total, Lp;
};
constexpr int kPairJobBytes = 128;   // the band's pair descriptor (PairJob) in shared memory
LUMEN_PAIR_HD PairSmem pair_smem(int Lmax, int Dp, int R) {
    PairSmem s;
    s.Lp = (Lmax + 15) & ~15;
    const int SB = pair_slot_bytes(Dp);
    int o = 0;
    s.img = o;
    o += (R + 1) * s.Lp;
    o = (o + 127) & ~127;
    s.cost = o;
    o += R * kPPF * Dp;
    s.slots = o;
    o += R * 2 * SB;
    s.imp = o;
    o += kPQ * SB;
    s.zero = o;   // all-zero slot: a path that starts reads it (L' = 0, min L' = 0 gives L = C)
    o += SB;
    s.lut = o;
    o += 256 * 4;
    s.job = o;
    o += kPairJobBytes;
    s.misc = o;
    o += 32 * 4;
    s.total = o;
    return s;
}

// sweep s, sweep coordinates (u, v) -> image (x, y)
LUMEN_PAIR_HD void pair_xy(int s, int u, int v, int W, int H, int& x, int& y) {
    if (s == 0) { x = u; y = v; }
    else if (s == 1) { x = W - 1 - u; y = H - 1 - v; }
    else if (s == 2) { x = W - 1 - v; y = u; }
    else { x = v; y = H - 1 - u; }
}

// ticket -> (sweep, band): the four sweeps round-robin while all have bands
// left, then the two sweeps with more bands alternate; every band comes
// after the band before it in its own sweep.
LUMEN_PAIR_HD void pair_ticket(int t, int nb0, int nb1, int& s, int& b) {
    const int m = nb0 < nb1 ? nb0 : nb1;
    if (t < 4 * m) {
        s = t & 3;
        b = t >> 2;
        return;
    }
    const int t2 = t - 4 * m;
    s = (nb0 > nb1 ? 0 : 2) + (t2 & 1);
    b = m + (t2 >> 1);
}

// first pixel (in row-buffer slots) of the row buffer of sweep s, boundary b
// (the last row of band b)
LUMEN_PAIR_HD size_t pair_xbase(int s, int b, int W, int H, int nb0, int nb1) {
    const size_t rows = (size_t)nb0 * W;
    if (s == 0) return (size_t)b * W;
    if (s == 1) return rows + (size_t)b * W;
    if (s == 2) return 2 * rows + (size_t)b * H;
    return 2 * rows + (size_t)nb1 * H + (size_t)b * H;
}

}  // namespace lumen
