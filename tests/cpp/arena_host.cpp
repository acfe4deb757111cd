// CPU test of the serving loop's tree placement (csrc/arena.h): first fit
// with coalescing, and eviction in least-recently-used order until a tree
// fits. Prints "ok" and exits 0, or names the failed check and exits 1.
#include <cstdio>
#include <map>
#include <vector>

#include "arena.h"

using frep::serving::Arena;
using frep::serving::LruOrder;
using frep::serving::place_evicting;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
            failures++;                                            \
        }                                                          \
    } while (0)

int main() {
    const uint64_t K = 256;
    {  // first fit, rounding, coalescing with both neighbours
        Arena a;
        a.reset(16 * K);
        uint64_t o1, o2, o3, o4;
        CHECK(a.alloc(1, &o1) && o1 == 0);          // rounded up to 256
        CHECK(a.alloc(2 * K, &o2) && o2 == K);
        CHECK(a.alloc(K + 1, &o3) && o3 == 3 * K);  // 512
        CHECK(a.used() == 5 * K);
        CHECK(a.release(o2, 2 * K) == 2 * K);       // between two used blocks
        CHECK(a.alloc(K, &o4) && o4 == K);          // first fit takes the hole
        CHECK(a.release(o4, K) == 2 * K);           // merges with the rest of the hole
        CHECK(a.release(o1, K) == 3 * K);           // merges with the next free block
        CHECK(a.release(o3, 2 * K) == 16 * K);      // both neighbours: everything is free
        CHECK(a.used() == 0 && a.free_blocks() == 1);
        uint64_t big;
        CHECK(!a.alloc(17 * K, &big));
    }
    {  // eviction order, kept entries, placement in the block an eviction grows
        Arena a;
        a.reset(8 * K);
        std::map<uint64_t, std::pair<uint64_t, uint64_t>> where;  // id -> (offset, bytes)
        LruOrder lru;
        uint64_t tick = 0;
        auto add = [&](uint64_t id, uint64_t bytes) {
            uint64_t off;
            if (!a.alloc(bytes, &off)) return false;
            where[id] = {off, bytes};
            lru.insert({++tick, id});
            return true;
        };
        std::vector<uint64_t> evicted;
        auto evict = [&](uint64_t id) {
            for (auto it = lru.begin(); it != lru.end(); ++it)
                if (it->second == id) {
                    lru.erase(it);
                    break;
                }
            evicted.push_back(id);
            const auto w = where[id];
            where.erase(id);
            return a.release(w.first, w.second);
        };
        // ids 1..8, one block each, oldest first
        for (uint64_t id = 1; id <= 8; id++) CHECK(add(id, K));
        // touch 1 and 2: they become the most recent
        for (uint64_t id : {1, 2}) {
            for (auto it = lru.begin(); it != lru.end(); ++it)
                if (it->second == id) {
                    lru.erase(it);
                    break;
                }
            lru.insert({++tick, id});
        }
        // a 2-block tree while 3 must stay: evicts 4, then 5 (adjacent: a 2-block hole)
        uint64_t off = 0;
        CHECK(place_evicting(a, lru, 2 * K, [](uint64_t id) { return id == 3; }, evict, &off));
        CHECK((evicted == std::vector<uint64_t>{4, 5}));
        CHECK(off == 3 * K);
        // nothing may be evicted and nothing fits: false, nothing evicted
        evicted.clear();
        CHECK(!place_evicting(a, lru, 4 * K, [](uint64_t) { return true; }, evict, &off));
        CHECK(evicted.empty());
        // the placed tree becomes id 9 (blocks 3-4), the most recent
        where[9] = {3 * K, 2 * K};
        lru.insert({++tick, 9});
        // a 3-block tree while 9 stays: evicts 3 (block 2, alone), then 6, 7, 8
        // (blocks 5-7 merge to 3) and is placed there; 1 and 2 are not touched
        CHECK(place_evicting(a, lru, 3 * K, [](uint64_t id) { return id == 9; }, evict, &off));
        CHECK((evicted == std::vector<uint64_t>{3, 6, 7, 8}));
        CHECK(off == 5 * K);
        CHECK(lru.size() == 3 && a.used() == 7 * K);
    }
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
