// Host model of schedule 6's hand-off protocol (pair_kernel.cuh) with the
// kernel's own ticket order, row-buffer layout and ring sizes (pair_layout.h).
// A worker thread stands for a resident CTA: it takes tickets from a shared
// counter and runs each band as two threads, the rows and the import warp.
//  * the band's last row writes, for every pixel u, the pixel's words into
//    the boundary row buffer as 64-bit (payload, epoch) words with relaxed
//    stores and no fence;
//  * the import warp takes the pixels 0 .. len-2 of the band above: it polls
//    up to kPG pixels at a time, copies the leading pixels whose words all
//    carry the launch's epoch into a kPQ-slot ring, never overwriting a slot
//    row 0 has not consumed, and publishes the count (release);
//  * row 0 at step u waits (bounded) for pixel u-1, reads it from the ring,
//    and after the step publishes how many pixels it has consumed.
// The row buffers hold stale words of an earlier launch (epoch - 1) at the
// start.  With any number of workers, from one to more than there are bands,
// every band must finish, and row 0 must only ever see the band above's
// words of this launch, in order.  Prints "ok" and exits 0 on success.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "pair_layout.h"

using namespace lumen;

static bool run(int W, int H, int R, int workers, unsigned seed) {
    const int nb0 = (H + R - 1) / R, nb1 = (W + R - 1) / R, nT = 2 * nb0 + 2 * nb1;
    const int NLW = 3;   // words a pixel in this model
    const uint32_t epoch = 7;
    std::vector<std::atomic<uint64_t>> xbuf(pair_xbase(3, nb1, W, H, nb0, nb1) * NLW);
    for (auto& x : xbuf) x.store((uint64_t)(epoch - 1) << 32 | 0xDEADu);   // a previous launch's words
    std::atomic<int> ticket{0}, failures{0};
    auto payload = [](int s, int b, int u, int w) -> uint32_t {
        return (uint32_t)(s * 7919 + b * 104729 + u * 31 + w * 1000003) & 0x7FFFFFFFu;
    };
    auto worker = [&](unsigned wseed) {
        std::mt19937 rng(wseed);
        for (;;) {
            const int t = ticket.fetch_add(1);
            if (t >= nT) return;
            int s, b;
            pair_ticket(t, nb0, nb1, s, b);
            const int Ws = s < 2 ? W : H, nb = s < 2 ? nb0 : nb1;
            const bool hasPrev = b > 0, hasNext = b + 1 < nb;
            const size_t xin = hasPrev ? pair_xbase(s, b - 1, W, H, nb0, nb1) * NLW : 0;
            const size_t xout = hasNext ? pair_xbase(s, b, W, H, nb0, nb1) * NLW : 0;
            std::vector<uint32_t> ring((size_t)kPQ * NLW);
            std::atomic<unsigned> imported{0}, consumed{0};
            std::atomic<bool> abort{false};
            std::thread importer([&] {
                if (!hasPrev) return;
                const int nImp = Ws - 1;
                int p0 = 0;
                long spins = 0;
                std::mt19937 irng(wseed ^ 0x9E3779B9u);
                while (p0 < nImp) {
                    const int g = std::min(kPG, nImp - p0);
                    while (p0 + g > kPQ && consumed.load(std::memory_order_acquire) < (unsigned)(p0 + g - kPQ)) {
                        if (abort.load() || ++spins > 200000000L) { failures++; abort = true; return; }
                        std::this_thread::yield();
                    }
                    uint64_t v[kPG][3];
                    int n = g;
                    for (int px = 0; px < g; ++px)
                        for (int w = 0; w < NLW; ++w) {
                            v[px][w] = xbuf[xin + (size_t)(p0 + px) * NLW + w].load(std::memory_order_relaxed);
                            if ((uint32_t)(v[px][w] >> 32) != epoch && px < n) n = px;
                        }
                    if (n == 0) {
                        if (abort.load() || ++spins > 200000000L) { failures++; abort = true; return; }
                        std::this_thread::yield();
                        continue;
                    }
                    for (int px = 0; px < n; ++px)
                        for (int w = 0; w < NLW; ++w)
                            ring[(size_t)((p0 + px) & (kPQ - 1)) * NLW + w] = (uint32_t)v[px][w];
                    imported.store((unsigned)(p0 + n), std::memory_order_release);
                    p0 += n;
                    spins = 0;
                    if ((irng() & 255) == 0) std::this_thread::yield();
                }
            });
            // the rows (row 0 consumes, the last row produces)
            for (int u = 0; u < Ws && !abort.load(); ++u) {
                if (hasPrev && u >= 1) {
                    long spins = 0;
                    while (imported.load(std::memory_order_acquire) < (unsigned)u) {
                        if (abort.load() || ++spins > 200000000L) { failures++; abort = true; break; }
                        std::this_thread::yield();
                    }
                    if (abort.load()) break;
                    for (int w = 0; w < NLW; ++w)
                        if (ring[(size_t)((u - 1) & (kPQ - 1)) * NLW + w] != payload(s, b - 1, u - 1, w)) failures++;
                }
                if (hasNext)
                    for (int w = 0; w < NLW; ++w)
                        xbuf[xout + (size_t)u * NLW + w].store((uint64_t)epoch << 32 | payload(s, b, u, w),
                                                               std::memory_order_relaxed);
                if (hasPrev) consumed.store((unsigned)u, std::memory_order_release);
                if ((rng() & 1023) == 0) std::this_thread::yield();   // uneven progress
            }
            importer.join();
        }
    };
    std::vector<std::thread> ts;
    for (int i = 0; i < workers; ++i) ts.emplace_back(worker, seed + i);
    for (auto& t : ts) t.join();
    if (failures.load()) return false;
    // every boundary row holds this launch's words for every pixel
    for (int s = 0; s < 4; ++s) {
        const int nb = s < 2 ? nb0 : nb1, Ws = s < 2 ? W : H;
        for (int b = 0; b + 1 < nb; ++b)
            for (int u = 0; u < Ws; ++u)
                for (int w = 0; w < NLW; ++w)
                    if (xbuf[pair_xbase(s, b, W, H, nb0, nb1) * NLW + (size_t)u * NLW + w].load() !=
                        ((uint64_t)epoch << 32 | payload(s, b, u, w)))
                        return false;
    }
    return true;
}

int main() {
    std::mt19937 rng(5);
    for (int it = 0; it < 40; ++it) {
        const int W = 1 + (int)(rng() % 300), H = 1 + (int)(rng() % 300);
        const int R = (it & 1) ? 32 : 16;
        const int workers = 1 + (int)(rng() % 12);
        if (!run(W, H, R, workers, rng())) {
            std::printf("FAILED W=%d H=%d R=%d workers=%d\n", W, H, R, workers);
            return 1;
        }
    }
    std::printf("ok\n");
    return 0;
}
