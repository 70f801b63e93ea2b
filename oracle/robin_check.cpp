// Check of the robin_hood iteration-order restatement — TEST INFRASTRUCTURE ONLY.
//
// Inserts seeded random integer sequences (small and large tables, runs with
// clear() in between, clustered keys that force long probe runs) into
// robin_hood::unordered_set<int> and unordered_map<int, std::vector<int>> from
// InstantGR's vendored src/robin_hood.h, and into igr::RobinOrder
// (instantgr_b200/csrc/robin_order.hpp), and compares the iteration orders.
// Prints "robin_check: <cases> cases, <mismatches> mismatches".
#include "robin_hood.h"
#include "robin_order.hpp"

#include <cstdint>
#include <cstdio>
#include <vector>

namespace {

int key_of(int k) { return k; }
template <class P>
int key_of(const P &p) { return p.first; }

uint64_t rng_state = 0x9E3779B97F4A7C15ULL;
uint64_t rnd() {
    uint64_t z = (rng_state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// keys whose home slot is 0 in every table of up to 2^bits buckets under the
// first hash multiplier: they pile up in one run, which drives the info bytes
// to overflow (halved increments, a new multiplier, growth)
int colliding_key(int bits) {
    for (;;) {
        const int k = (int)(rnd() & 0x3fffffff);
        uint64_t h = (uint64_t)(int64_t)k;
        h ^= h >> 33;
        h *= 0xff51afd7ed558ccdULL;
        h ^= h >> 33;
        h *= 0xc4ceb9fe1a85ec53ULL;
        h ^= h >> 33;
        if (((h >> 5) & ((1ULL << bits) - 1)) == 0) return k;
    }
}

template <class Ref>
bool same(const Ref &ref, const igr::RobinOrder &mine) {
    std::vector<int> a, b;
    for (auto &e : ref) a.push_back(key_of(e));
    mine.for_each([&](int k) { b.push_back(k); });
    return a == b;
}

}  // namespace

int main() {
    long cases = 0, bad = 0;
    for (int t = 0; t < 4000; t++) {
        const int runs = 1 + (int)(rnd() % 3);
        robin_hood::unordered_set<int> rs;
        robin_hood::unordered_map<int, std::vector<int>> rm;
        igr::RobinOrder ms, mm;
        for (int r = 0; r < runs; r++) {
            const int n = (int)(t % 7 == 0 ? rnd() % 20000 : rnd() % 300);
            const int mode = (int)(rnd() % 5);
            const int range = mode == 0 ? 50 : (mode == 1 ? 1000 : (mode == 2 ? 1 << 30 : 4 * (n + 1)));
            for (int i = 0; i < n; i++) {
                int k = mode == 3 ? (int)(i * 4096) : (int)(rnd() % (uint64_t)range);
                if (mode == 4) k = (i % 3 == 0) ? colliding_key(3 + (int)(rnd() % 8)) : (int)(rnd() % 100000);
                if (mode == 2 && (rnd() & 1)) k = -k;
                rs.insert(k);
                ms.insert(k);
                rm[k].push_back(i);
                mm.insert(k);
            }
            cases++;
            if (!same(rs, ms) || !same(rm, mm) || rs.size() != ms.size()) {
                bad++;
                if (bad < 5) std::printf("mismatch: case %d run %d n %d mode %d\n", t, r, n, mode);
            }
            rs.clear();
            rm.clear();
            ms.clear();
            mm.clear();
        }
    }
    std::printf("robin_check: %ld cases, %ld mismatches\n", cases, bad);
    return bad ? 1 : 0;
}
