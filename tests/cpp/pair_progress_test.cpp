// Host model of schedule 6's hand-off protocol (pair_kernel.cuh) with the
// kernel's own ticket order and counter layout (pair_layout.h): worker
// threads stand for resident CTAs, take tickets from a shared counter, and
// run their band pixel by pixel; a band with a predecessor waits (bounded)
// until the band above has published pixel u before using it one step later,
// and the band's last row publishes its progress every kPE pixels and at the
// end (release / acquire).  With any number of workers, from one to more
// than there are bands, every band must finish and must only ever consume
// pixels its predecessor had published.  Prints "ok" and exits 0 on success.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "pair_layout.h"

using namespace lumen;

static bool run(int W, int H, int workers, unsigned seed) {
    const int R = 16;
    const int nb0 = (H + R - 1) / R, nb1 = (W + R - 1) / R, nT = 2 * nb0 + 2 * nb1;
    std::vector<std::atomic<unsigned>> prod(nT);
    for (auto& p : prod) p.store(0);
    // the row buffers: the value a band's last row wrote at each pixel
    std::vector<std::atomic<int>> xbuf(pair_xbase(3, nb1, W, H, nb0, nb1));
    for (auto& x : xbuf) x.store(-1);
    std::atomic<int> ticket{0}, failures{0};
    auto worker = [&](unsigned wseed) {
        std::mt19937 rng(wseed);
        for (;;) {
            const int t = ticket.fetch_add(1);
            if (t >= nT) return;
            int s, b;
            pair_ticket(t, nb0, nb1, s, b);
            const int Ws = s < 2 ? W : H, nb = s < 2 ? nb0 : nb1;
            const bool hasPrev = b > 0, hasNext = b + 1 < nb;
            const int pin = pair_poff(s, nb0, nb1) + b - 1, pout = pair_poff(s, nb0, nb1) + b;
            const size_t xin = hasPrev ? pair_xbase(s, b - 1, W, H, nb0, nb1) : 0;
            const size_t xout = hasNext ? pair_xbase(s, b, W, H, nb0, nb1) : 0;
            int pred = -1;   // the band above's pixel u-1, loaded during step u-1
            for (int u = 0; u < Ws; ++u) {
                int cur = pred;
                if (hasPrev && u + 1 < Ws) {
                    // bounded wait for pixel u, then load it for the next step
                    long spins = 0;
                    while (prod[pin].load(std::memory_order_acquire) < (unsigned)(u + 1)) {
                        if (++spins > 200000000L) { failures++; return; }
                        std::this_thread::yield();
                    }
                    pred = xbuf[xin + u].load(std::memory_order_relaxed);
                    if (pred != u) failures++;   // consumed before it was written
                }
                if (hasPrev && u > 0 && cur != u - 1) failures++;
                if (hasNext) xbuf[xout + u].store(u, std::memory_order_relaxed);
                if (hasNext && ((u % kPE) == kPE - 1 || u == Ws - 1))
                    prod[pout].store((unsigned)(u + 1), std::memory_order_release);
                if ((rng() & 1023) == 0) std::this_thread::yield();   // uneven progress
            }
        }
    };
    std::vector<std::thread> ts;
    for (int i = 0; i < workers; ++i) ts.emplace_back(worker, seed + i);
    for (auto& t : ts) t.join();
    if (failures.load()) return false;
    for (int s = 0; s < 4; ++s) {
        const int nb = s < 2 ? nb0 : nb1, Ws = s < 2 ? W : H;
        for (int b = 0; b + 1 < nb; ++b)
            if (prod[pair_poff(s, nb0, nb1) + b].load() != (unsigned)Ws) return false;
    }
    return true;
}

int main() {
    std::mt19937 rng(5);
    for (int it = 0; it < 40; ++it) {
        const int W = 1 + (int)(rng() % 300), H = 1 + (int)(rng() % 300);
        const int workers = 1 + (int)(rng() % 12);
        if (!run(W, H, workers, rng())) {
            std::printf("FAILED W=%d H=%d workers=%d\n", W, H, workers);
            return 1;
        }
    }
    std::printf("ok\n");
    return 0;
}
