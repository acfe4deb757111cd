// Host-side placement of the serving loop's resident trees (frep_server): one
// device allocation carved first fit, and eviction in least-recently-used
// order until a new tree fits. Plain C++ (no CUDA), so that the policy is
// tested on the CPU (tests/cpp/arena_host.cpp).
#pragma once

#include <cstdint>
#include <iterator>
#include <map>
#include <set>
#include <utility>

namespace frep {
namespace serving {

inline uint64_t align_256(uint64_t v) { return (v + 255u) / 256u * 256u; }

// First fit over one allocation of `bytes`, with coalescing of free
// neighbours. Sizes are rounded up to 256 bytes.
class Arena {
   public:
    void reset(uint64_t bytes) {
        free_.clear();
        free_[0] = bytes;
        cap_ = bytes;
        used_ = 0;
    }
    bool alloc(uint64_t bytes, uint64_t* off) {
        bytes = align_256(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const uint64_t rest = it->second - bytes;
            const uint64_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    // Returns the size of the free block that now holds [off, off + bytes).
    uint64_t release(uint64_t off, uint64_t bytes) {
        bytes = align_256(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
                return prev->second;
            }
        }
        return it->second;
    }
    uint64_t used() const { return used_; }
    uint64_t capacity() const { return cap_; }
    size_t free_blocks() const { return free_.size(); }

   private:
    std::map<uint64_t, uint64_t> free_;  // offset -> bytes
    uint64_t cap_ = 0, used_ = 0;
};

// Resident entries by (last use, id): begin() is the least recently used.
using LruOrder = std::set<std::pair<uint64_t, uint64_t>>;

// Places `bytes` in `arena`, evicting entries of `lru` from the least
// recently used on until a free block holds them. keep(id): an entry that
// must stay (the trees of the step being formed; they carry the newest use
// and come last). evict(id): releases the entry's memory, removes it from
// `lru`, and returns the size of the free block that now holds that memory.
// Only the block an eviction grows can newly fit `bytes`, so first fit runs
// again only when that block is large enough. False: nothing more can be
// evicted and `bytes` still does not fit.
template <class Keep, class Evict>
bool place_evicting(Arena& arena, const LruOrder& lru, uint64_t bytes, Keep keep, Evict evict, uint64_t* off) {
    if (arena.alloc(bytes, off)) return true;
    const uint64_t need = align_256(bytes);
    for (;;) {
        auto it = lru.begin();
        while (it != lru.end() && keep(it->second)) ++it;
        if (it == lru.end()) return false;
        if (evict(it->second) >= need && arena.alloc(bytes, off)) return true;
    }
}

}  // namespace serving
}  // namespace frep
