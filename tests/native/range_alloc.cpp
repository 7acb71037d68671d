// Host test driver for kpolaris_b200/csrc/kp_range_alloc.h: a seeded random
// sequence of allocations and releases checked against a bitmap model
// (no overlap, every free unit reachable after coalescing).  Prints "ok".
#include <cstdio>
#include <random>
#include <vector>

#include "kp_range_alloc.h"

int main() {
    const long long cap = 4096;
    kp::RangeAllocator a(cap);
    std::vector<int> owner(cap, -1);
    struct Live { long long s, n; };
    std::vector<Live> live;
    std::mt19937 rng(7);
    for (int step = 0; step < 20000; ++step) {
        if (!live.empty() && (rng() % 3 == 0 || a.largest_free() == 0)) {
            const size_t k = rng() % live.size();
            for (long long u = live[k].s; u < live[k].s + live[k].n; ++u) owner[u] = -1;
            a.release(live[k].s, live[k].n);
            live.erase(live.begin() + long(k));
        } else {
            const long long n = 1 + rng() % 300;
            const long long s = a.alloc(n);
            if (s < 0) {
                if (a.largest_free() >= n) { std::printf("missed fit\n"); return 1; }
                continue;
            }
            for (long long u = s; u < s + n; ++u) {
                if (owner[u] != -1) { std::printf("overlap\n"); return 1; }
                owner[u] = step;
            }
            live.push_back({s, n});
        }
        long long used = 0;
        for (int o : owner) used += o != -1;
        if (used != a.used()) { std::printf("used mismatch\n"); return 1; }
    }
    for (const auto& l : live) a.release(l.s, l.n);
    if (a.used() != 0 || a.largest_free() != cap || a.fragments() != 1) { std::printf("not coalesced\n"); return 1; }
    std::printf("ok\n");
    return 0;
}
