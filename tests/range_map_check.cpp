// Randomised check of the scratch arena's range bookkeeping (range_map.h):
// best fit, no overlap, full coalescing, conservation of bytes.  Built and
// run by tests/test_range_map_cpu.py; exits non-zero on the first violation.
#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <random>
#include <vector>

#include "range_map.h"

#define CHECK(c)                                                    \
    do {                                                            \
        if (!(c)) {                                                 \
            fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
            return 1;                                               \
        }                                                           \
    } while (0)

int main() {
    std::mt19937_64 rng(0x5C4A7C4);
    for (int trial = 0; trial < 50; ++trial) {
        const size_t total = 1 + rng() % 100000;
        gpupi::RangeMap m;
        m.reset(total);
        std::map<size_t, size_t> live;   // offset -> size
        for (int step = 0; step < 2000; ++step) {
            if (live.empty() || rng() % 3 != 0) {
                const size_t want = 1 + rng() % (1 + total / 8);
                size_t best = 0;
                bool any = false;
                for (auto &r : m.ranges())
                    if (r.second >= want && (!any || r.second < best)) best = r.second, any = true;
                const std::map<size_t, size_t> before = m.ranges();
                size_t off = 0;
                const bool got = m.take(want, &off);
                CHECK(got == any);
                if (!got) continue;
                CHECK(off + want <= total);
                auto nx = live.lower_bound(off);
                CHECK(nx == live.end() || off + want <= nx->first);
                if (nx != live.begin()) {
                    auto pv = std::prev(nx);
                    CHECK(pv->first + pv->second <= off);
                }
                // it came from the start of a smallest fitting free range
                CHECK(before.count(off) == 1 && before.at(off) == best);
                live[off] = want;
            } else {
                auto it = live.begin();
                std::advance(it, rng() % live.size());
                m.give(it->first, it->second);
                live.erase(it);
            }
            size_t free_bytes = 0, live_bytes = 0, end = 0;
            bool first = true;
            for (auto &r : m.ranges()) {
                CHECK(r.second > 0);
                CHECK(first || r.first > end);   // sorted, disjoint, never adjacent
                end = r.first + r.second;
                CHECK(end <= total);
                free_bytes += r.second;
                first = false;
                auto nx = live.lower_bound(r.first);   // no live block inside a free range
                CHECK(nx == live.end() || nx->first >= end);
            }
            for (auto &l : live) live_bytes += l.second;
            CHECK(free_bytes + live_bytes == total);
        }
        for (auto &l : live) m.give(l.first, l.second);
        CHECK(m.free_ranges() == 1);
        CHECK(m.ranges().begin()->first == 0 && m.ranges().begin()->second == total);
    }
    // best fit: of free ranges 10 and 6, a request of 5 takes the 6
    gpupi::RangeMap m;
    m.reset(30);
    size_t a, b, c, d;
    CHECK(m.take(10, &a) && m.take(4, &b) && m.take(6, &c) && m.take(10, &d));
    m.give(a, 10);
    m.give(c, 6);
    size_t e;
    CHECK(m.take(5, &e) && e == c);
    printf("range_map ok\n");
    return 0;
}
