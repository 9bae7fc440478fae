// Checks of schedule 6's shared index arithmetic (pair_layout.h), the
// properties the kernel's correctness and progress rest on:
//  * every (sweep, band) gets exactly one ticket, and within a sweep the bands
//    come in order (a band only waits on the band above it, an earlier ticket);
//  * each sweep visits every pixel once, and the predecessor of its
//    horizontal and diagonal path is the reference path's previous pixel
//    (LR/TLBR, RL/BRTL, TB/TRBL, BT/BLTR);
//  * band-boundary row buffers never overlap and stay inside the size the
//    host allocates;
//  * the shared-memory carve-up and the row-buffer words keep the cp.async
//    and vector alignments.
// Prints "ok" and exits 0 on success.
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "pair_layout.h"

using namespace lumen;

#define CHECK(c)                                                      \
    do {                                                              \
        if (!(c)) {                                                   \
            std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c); \
            return 1;                                                 \
        }                                                             \
    } while (0)

int main() {
    const int R = 16;
    std::mt19937_64 rng(11);
    // tickets, row buffers, counters
    for (int it = 0; it < 4000; ++it) {
        const int W = 1 + (int)(rng() % 6000), H = 1 + (int)(rng() % 6000);
        const int nb0 = (H + R - 1) / R, nb1 = (W + R - 1) / R;
        const int nT = 2 * nb0 + 2 * nb1;
        std::vector<int> last(4, -1);
        std::vector<int> count(4, 0);
        for (int t = 0; t < nT; ++t) {
            int s, b;
            pair_ticket(t, nb0, nb1, s, b);
            CHECK(s >= 0 && s < 4);
            CHECK(b == last[s] + 1);   // in order, each band once
            last[s] = b;
            ++count[s];
        }
        CHECK(count[0] == nb0 && count[1] == nb0 && count[2] == nb1 && count[3] == nb1);
        const size_t total = pair_xbase(3, nb1, W, H, nb0, nb1);
        size_t prev = 0;
        for (int s = 0; s < 4; ++s) {
            const int nb = s < 2 ? nb0 : nb1, Ws = s < 2 ? W : H;
            for (int b = 0; b < nb; ++b) {
                const size_t x0 = pair_xbase(s, b, W, H, nb0, nb1);
                CHECK(x0 == prev);       // consecutive, disjoint
                prev = x0 + (size_t)Ws;
                CHECK(prev <= total);
            }
        }
        CHECK(prev == total);
    }
    // geometry: bijection and path predecessors
    const int dH[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};     // LR, RL, TB, BT
    const int dD[4][2] = {{-1, -1}, {1, 1}, {1, -1}, {-1, 1}};   // TLBR, BRTL, TRBL, BLTR
    for (int it = 0; it < 300; ++it) {
        const int W = 1 + (int)(rng() % 40), H = 1 + (int)(rng() % 40);
        for (int s = 0; s < 4; ++s) {
            const int Ws = s < 2 ? W : H, Hs = s < 2 ? H : W;
            std::set<std::pair<int, int>> seen;
            for (int v = 0; v < Hs; ++v)
                for (int u = 0; u < Ws; ++u) {
                    int x, y;
                    pair_xy(s, u, v, W, H, x, y);
                    CHECK(x >= 0 && x < W && y >= 0 && y < H);
                    CHECK(seen.insert({x, y}).second);
                    if (u > 0) {
                        int px, py;
                        pair_xy(s, u - 1, v, W, H, px, py);
                        CHECK(px == x + dH[s][0] && py == y + dH[s][1]);
                        if (v > 0) {
                            pair_xy(s, u - 1, v - 1, W, H, px, py);
                            CHECK(px == x + dD[s][0] && py == y + dD[s][1]);
                        }
                    }
                    // the path starts exactly where its predecessor leaves the image
                    const int hx = x + dH[s][0], hy = y + dH[s][1];
                    CHECK((u == 0) == !(hx >= 0 && hx < W && hy >= 0 && hy < H));
                    const int qx = x + dD[s][0], qy = y + dD[s][1];
                    CHECK((u == 0 || v == 0) == !(qx >= 0 && qx < W && qy >= 0 && qy < H));
                }
            CHECK((int)seen.size() == W * H);
        }
    }
    // shared memory: alignments of the cost ring (cp.async 16 B), slots, import
    // ring and zero slot; row-buffer words: every pixel starts on 16 bytes and
    // the import warp's 8-byte pairs land inside a slot
    for (int Dp : {64, 128, 192, 256, 320}) {
        CHECK(pair_ll_words(Dp) % 2 == 0 && pair_ll_words(Dp) >= Dp / 2 + 1);
        CHECK(8 * (pair_ll_words(Dp) / 2) <= pair_slot_bytes(Dp));   // 8-byte pairs of payload into a slot
        CHECK(4 * (Dp / 2) == 2 * Dp);                               // the minimum's word sits at byte 2 Dp
        for (int RR : {16, 32})
            for (int L = 1; L < 8000; L += 37) {
                const PairSmem m = pair_smem(L, Dp, RR);
                CHECK(m.Lp >= L && m.Lp % 16 == 0);
                CHECK(m.cost % 128 == 0 && m.cost >= (RR + 1) * L);
                CHECK(m.slots % 16 == 0 && m.imp % 16 == 0 && m.zero % 16 == 0 && m.lut % 4 == 0 &&
                      m.job % 16 == 0 && m.misc % 4 == 0);
                CHECK(m.misc - m.job == kPairJobBytes);
                CHECK(m.imp - m.slots == RR * 2 * pair_slot_bytes(Dp));
                CHECK(m.zero - m.imp == kPQ * pair_slot_bytes(Dp));
                CHECK(pair_slot_bytes(Dp) % 16 == 0);
                CHECK(m.total == m.misc + 128);
            }
    }
    std::printf("ok\n");
    return 0;
}
