// host_arena.h -- the served form's device-arena bookkeeping (host only):
// first-fit allocation of byte ranges of a fixed-size arena, 256-byte units,
// adjacent free ranges coalesced on release.
#pragma once
#include <cstddef>
#include <iterator>
#include <map>

namespace lumen {

class Arena {
  public:
    void reset(size_t size) {
        free_.clear();
        if (size) free_[0] = size;
    }
    bool alloc(size_t n, size_t* off) {
        n = (n + 255) & ~size_t(255);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                const size_t rest = it->second - n, at = it->first + n;
                free_.erase(it);
                if (rest) free_[at] = rest;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n) {
        n = (n + 255) & ~size_t(255);
        auto next = free_.lower_bound(off);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            free_.erase(next);
        }
        free_[off] = n;
    }
    size_t free_bytes() const {
        size_t n = 0;
        for (auto& kv : free_) n += kv.second;
        return n;
    }
    size_t free_blocks() const { return free_.size(); }

  private:
    std::map<size_t, size_t> free_;  // offset -> length
};

}  // namespace lumen
