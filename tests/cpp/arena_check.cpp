// CPU check of the request loop's device-range allocator (serve_arena.hpp):
// first fit, alignment, coalescing on release, peak tracking, exhaustion.
// Prints "ok" and exits 0 when every check holds.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../hpc_ode_b200/csrc/serve_arena.hpp"

#define CHECK(c)                                                 \
    do {                                                         \
        if (!(c)) {                                              \
            std::printf("FAILED line %d: %s\n", __LINE__, #c);   \
            return 1;                                            \
        }                                                        \
    } while (0)

int main() {
    using b200::RangeArena;
    RangeArena a(10000);
    CHECK(a.capacity() == 9984);   // rounded down to 256
    size_t o1, o2, o3, o4;
    CHECK(a.alloc(1, &o1) && o1 == 0);
    CHECK(a.alloc(300, &o2) && o2 == 256);
    CHECK(a.alloc(256, &o3) && o3 == 768);
    CHECK(a.used() == 1024);
    CHECK(!a.alloc(9000, &o4));                 // does not fit
    a.release(o2, 300);                         // hole of 512 at 256
    CHECK(a.alloc(400, &o4) && o4 == 256);      // first fit reuses the hole
    a.release(o4, 400);
    a.release(o1, 1);
    a.release(o3, 256);
    CHECK(a.used() == 0 && a.free_ranges() == 1 && a.largest_free() == 9984);   // fully coalesced
    CHECK(a.peak() == 1024);

    // random alloc/release against a shadow map of occupied bytes
    std::mt19937_64 rng(5);
    RangeArena b(1 << 20);
    std::vector<std::pair<size_t, size_t>> live;
    std::vector<unsigned char> owner(1 << 20, 0);
    for (int it = 0; it < 20000; ++it) {
        if (!live.empty() && (rng() % 2)) {
            const size_t k = rng() % live.size();
            const size_t off = live[k].first, len = RangeArena::round_up(live[k].second);
            for (size_t i = off; i < off + len; ++i) owner[i] = 0;
            b.release(live[k].first, live[k].second);
            live.erase(live.begin() + k);
        } else {
            const size_t sz = 1 + rng() % 40000;
            size_t off;
            if (b.alloc(sz, &off)) {
                CHECK(off % 256 == 0 && off + RangeArena::round_up(sz) <= b.capacity());
                for (size_t i = off; i < off + RangeArena::round_up(sz); ++i) {
                    CHECK(owner[i] == 0);      // never overlaps a live range
                    owner[i] = 1;
                }
                live.emplace_back(off, sz);
            }
        }
        size_t used = 0;
        for (auto& l : live) used += RangeArena::round_up(l.second);
        CHECK(used == b.used());
    }
    for (auto& l : live) b.release(l.first, l.second);
    CHECK(b.used() == 0 && b.free_ranges() == 1);
    std::printf("ok\n");
    return 0;
}
