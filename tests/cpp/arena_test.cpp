// Randomised check of the served form's arena bookkeeping (host_arena.h):
// live ranges never overlap and stay inside the arena, a request that fits
// the largest free range is granted, and freeing everything coalesces the
// arena back into one range.  Prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "host_arena.h"

int main() {
    const size_t size = size_t(1) << 30;
    lumen::Arena a;
    a.reset(size);
    std::mt19937_64 rng(12345);
    struct Live { size_t off, n; };
    std::vector<Live> live;
    size_t used = 0;
    for (int it = 0; it < 200000; ++it) {
        if (live.empty() || rng() % 3) {
            const size_t n = 1 + rng() % (size / 64);
            size_t off = 0;
            if (a.alloc(n, &off)) {
                const size_t r = (n + 255) & ~size_t(255);
                if (off % 256 || off + r > size) { std::printf("range outside the arena\n"); return 1; }
                for (const Live& l : live)
                    if (off < l.off + l.n && l.off < off + r) { std::printf("overlap\n"); return 1; }
                live.push_back({off, r});
                used += r;
            }
        } else {
            const size_t k = rng() % live.size();
            a.release(live[k].off, live[k].n);
            used -= live[k].n;
            live[k] = live.back();
            live.pop_back();
        }
        if (a.free_bytes() != size - used) { std::printf("free bytes %zu != %zu\n", a.free_bytes(), size - used); return 1; }
    }
    for (const Live& l : live) a.release(l.off, l.n);
    if (a.free_blocks() != 1 || a.free_bytes() != size) { std::printf("not coalesced\n"); return 1; }
    size_t off = 1;
    if (!a.alloc(size, &off) || off != 0) { std::printf("whole arena not grantable\n"); return 1; }
    std::printf("ok\n");
    return 0;
}
