// batch_tickets.h -- the ticket table of one batched sweep launch (host only).
//
// Every band of every pair of a group, both sweeps, as entries
// pair << 20 | sweep << 19 | band.  A band's import waits on the band above
// it (the previous band of its pair and sweep), and its export waits, through
// the ring back-pressure, on the next lookahead_bands(W) bands below it.  A
// CTA takes a ticket only while it runs, so the oldest unfinished ticket can
// finish whenever the tickets it needs are at most `window` positions later
// and window + 1 CTAs are resident.  Pairs are cut into chunks; tickets are
// band-major inside a chunk (the chunk's wavefronts overlap) and chunk after
// chunk, the chunks as large as the window allows.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace lumen {

// bands below a band that must run for it to finish a row of W pixels when
// the ring between two bands holds ringPixels pixels: a band with no CTA
// stalls the band above it after ringPixels pixels, that one after about
// twice as many, and so on (one more for the in-band row lag and the import
// queue)
inline int lookahead_bands(int W, int ringPixels) { return (W + ringPixels - 1) / ringPixels + 1; }

struct TicketPair {
    int W;       // image width (pixels per sweep row)
    int nBands;  // bands per sweep
};

// Fills `table`; returns the window, or -1 when one pair alone needs more
// than grid - 1 tickets of window (it cannot run on `grid` resident CTAs).
inline int build_ticket_table(const std::vector<TicketPair>& ps, int grid, int ringPixels,
                              std::vector<uint32_t>& table) {
    table.clear();
    int window = 0;
    for (int j0 = 0; j0 < (int)ps.size();) {
        int j1 = j0, Wc = 0, nb = 0;
        while (j1 < (int)ps.size()) {
            const int w2 = std::max(Wc, ps[j1].W);
            if (j1 > j0 && 2 * (j1 - j0 + 1) * lookahead_bands(w2, ringPixels) + 1 > grid) break;
            Wc = w2;
            nb = std::max(nb, ps[j1].nBands);
            ++j1;
        }
        int chunkTickets = 0;
        for (int j = j0; j < j1; ++j) chunkTickets += 2 * ps[j].nBands;
        // needs stay inside the chunk
        const int win = std::min(2 * (j1 - j0) * lookahead_bands(Wc, ringPixels), chunkTickets);
        if (win + 1 > grid) return -1;
        window = std::max(window, win);
        for (int band = 0; band < nb; ++band)
            for (int j = j0; j < j1; ++j)
                if (band < ps[j].nBands)
                    for (int sw = 0; sw < 2; ++sw)
                        table.push_back(((uint32_t)j << 20) | ((uint32_t)sw << 19) | (uint32_t)band);
        j0 = j1;
    }
    return window;
}

}  // namespace lumen
