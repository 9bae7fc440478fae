// Randomised check of the batched sweep launch's ticket table
// (batch_tickets.h), the property its progress rests on: every band of every
// pair and sweep appears once, after the band above it, and every band the
// ring back-pressure can make it wait for (the next lookahead_bands(W) bands
// of its pair and sweep) is at most `window` tickets later, with window + 1 no
// more than the resident CTAs.  Prints "ok" and exits 0 on success.
#include <cstdio>
#include <map>
#include <random>
#include <tuple>
#include <vector>

#include "batch_tickets.h"

int main() {
    std::mt19937_64 rng(7);
    const int ring = 256;
    int cases = 0;
    for (int it = 0; it < 3000; ++it) {
        const int n = 1 + (int)(rng() % 64);
        const int grid = 8 + (int)(rng() % 600);
        std::vector<lumen::TicketPair> ps(n);
        for (auto& p : ps) {
            p.W = 2 + (int)(rng() % 4096);
            p.nBands = 1 + (int)(rng() % 300);
        }
        std::vector<uint32_t> t;
        const int win = lumen::build_ticket_table(ps, grid, ring, t);
        if (win < 0) {  // only when one pair alone cannot fit
            bool single = false;
            for (auto& p : ps)
                single |= std::min(2 * lumen::lookahead_bands(p.W, ring), 2 * p.nBands) + 1 > grid;
            if (!single) { std::printf("refused a table that fits\n"); return 1; }
            continue;
        }
        ++cases;
        if (win + 1 > grid) { std::printf("window %d exceeds grid %d\n", win, grid); return 1; }
        std::map<std::tuple<int, int, int>, int> pos;
        size_t expect = 0;
        for (auto& p : ps) expect += 2 * (size_t)p.nBands;
        if (t.size() != expect) { std::printf("ticket count\n"); return 1; }
        for (int i = 0; i < (int)t.size(); ++i) {
            const int j = (int)(t[i] >> 20), sw = (int)((t[i] >> 19) & 1), b = (int)(t[i] & 0x7FFFFu);
            if (j >= n || b >= ps[j].nBands) { std::printf("entry out of range\n"); return 1; }
            if (!pos.emplace(std::make_tuple(j, sw, b), i).second) { std::printf("duplicate\n"); return 1; }
        }
        for (auto& kv : pos) {
            const int j = std::get<0>(kv.first), sw = std::get<1>(kv.first), b = std::get<2>(kv.first);
            const int i = kv.second;
            if (b > 0 && pos[std::make_tuple(j, sw, b - 1)] > i) { std::printf("band before its predecessor\n"); return 1; }
            const int L = lumen::lookahead_bands(ps[j].W, ring);
            for (int k = 1; k <= L && b + k < ps[j].nBands; ++k)
                if (pos[std::make_tuple(j, sw, b + k)] - i > win) {
                    std::printf("needed band %d tickets later, window %d\n", pos[std::make_tuple(j, sw, b + k)] - i, win);
                    return 1;
                }
        }
    }
    if (cases < 1000) { std::printf("too few cases\n"); return 1; }
    std::printf("ok\n");
    return 0;
}
