// Pin access-point selection: one access point per pin, restating the rules of
// InstantGR's net::init (src/database.hpp:38-243).
//
//  * <= 4 pins: every combination is enumerated (pin 0 varies slowest) and the
//    best is kept by (2-D mismatch count, bbox half-perimeter, distance to the
//    bbox centre, layer sum) with the reference's strict/equal tie rules
//    (src/database.hpp:46-97).
//  * > 4 pins: greedy rounds pick the 2-D position shared by the most
//    unvisited pins (running counts, then x/y coordinate repetition, then
//    centre distance), then every remaining pin takes its access point with the
//    most coordinate repetition (src/database.hpp:98-223).  The running counts
//    make the choice depend on the order in which the pins are walked: the
//    reference walks them in the iteration order of a robin_hood hash set
//    filled from a robin_hood hash map, and so do these rounds (RobinOrder,
//    robin_order.hpp).
//  * Pins that end up stacked on one 2-D position keep the highest one as the
//    pin and emit a via (lowest, highest) as an extra route
//    (src/database.hpp:225-242).
//  * The pins come out in the iteration order of the reference's robin_hood
//    sets of chosen positions (3-D, or 2-D when pins were stacked), the order in
//    which its later steps (the Steiner provider's input, the net split) see them.
#include "host.hpp"
#include "robin_order.hpp"

#include <algorithm>
#include <cstdint>

namespace igr {

namespace {

// Map of one net's non-negative keys to values (open addressing, linear
// probing); reset() empties it for the next net by a generation stamp.
class KeyIndex {
public:
    void reset(size_t expected) {
        size_t cap = 16;
        while (cap < 2 * expected) cap <<= 1;
        if (keys_.size() < cap) {
            keys_.assign(cap, 0);
            vals_.assign(cap, 0);
            gen_.assign(cap, 0);
            cur_ = 0;
        }
        mask_ = cap - 1;
        if (++cur_ == 0) {
            std::fill(gen_.begin(), gen_.end(), 0u);
            cur_ = 1;
        }
    }
    // value of `key`, inserting `val` when absent
    int find_or_insert(int key, int val) {
        for (size_t h = slot(key);; h = (h + 1) & mask_) {
            if (gen_[h] != cur_) {
                gen_[h] = cur_;
                keys_[h] = key;
                vals_[h] = val;
                return val;
            }
            if (keys_[h] == key) return vals_[h];
        }
    }
    int find(int key) const {
        for (size_t h = slot(key);; h = (h + 1) & mask_) {
            if (gen_[h] != cur_) return -1;
            if (keys_[h] == key) return vals_[h];
        }
    }

private:
    std::vector<int> keys_, vals_;
    std::vector<uint32_t> gen_;
    uint32_t cur_ = 0;
    size_t mask_ = 0;
    size_t slot(int key) const { return (size_t)(((uint64_t)(uint32_t)key * 0x9E3779B97F4A7C15ull) >> 40) & mask_; }
};

// Counts per grid column or row for one net at a time (a stamp per entry
// marks the counts of the current net).
struct StampedCounts {
    std::vector<int> val;
    std::vector<uint32_t> st;
    uint32_t cur = 0;
    void next(int n) {
        if ((int)val.size() < n) {
            val.assign(n, 0);
            st.assign(n, 0);
            cur = 0;
        }
        if (++cur == 0) {
            std::fill(st.begin(), st.end(), 0u);
            cur = 1;
        }
    }
    int get(int k) const { return st[k] == cur ? val[k] : 0; }
    void inc(int k) {
        if (st[k] != cur) { st[k] = cur; val[k] = 0; }
        val[k]++;
    }
};

struct PinScratch {
    std::vector<int> idx, best;
    std::vector<int> ax, ay, al, aoff;  // decoded access points of a net of at most 4 pins (pin-major)
    std::vector<int> kx, ky, kd;        // per 2-D key of a larger net: x, y, distance to the bbox centre (x2)
    std::vector<char> visited;
    std::vector<int> p, p2;
    std::vector<int> order;        // walk order of the pins in the greedy rounds
    RobinOrder keys2d, walk, rp, rp2;
    std::vector<int> first2d;      // 2-D keys of the access points in first-seen order
    KeyIndex rank;                 // 2-D key -> its index in first2d
    std::vector<int> ap_rank;      // per access point of the net (pin-major): rank of its 2-D key
    std::vector<int> list_off, list_pin;  // pins per 2-D key (CSR by rank, push order)
    std::vector<int> cnt;          // running count per 2-D key in the current round
    std::vector<uint32_t> cnt_st;  // round stamp of cnt
    uint32_t round_st = 0;
    std::vector<int> lst;          // pins at the chosen key in a round
    std::vector<int> mn, mx;       // lowest / highest chosen position per 2-D key
    StampedCounts xcnt, ycnt;
};

void select_one(const Design &d, int n, PinScratch &s, std::vector<int> &pins, std::vector<int> &extra) {
    const int X = d.X, Y = d.Y, XY = X * Y;
    const int64_t pb = d.pin_off[n];
    const int num = (int)(d.pin_off[n + 1] - pb);
    auto nap = [&](int i) { return (int)(d.ap_off[pb + i + 1] - d.ap_off[pb + i]); };
    auto apv = [&](int i, int j) { return d.ap[d.ap_off[pb + i] + j]; };  // j is 0-based
    const int c2x = d.bminx[n] + d.bmaxx[n], c2y = d.bminy[n] + d.bmaxy[n];
    std::vector<int> &p = s.p, &p2 = s.p2;  // chosen 3-D positions, chosen 2-D positions
    p.clear(); p2.clear();
    s.rp.reset(); s.rp2.reset();  // net::init's sets are declared anew for every net
    // the reference's robin_hood sets p and p2D (their insertion sequences);
    // p and p2 hold their elements in first-insertion order
    auto has2 = [&](int v) { return s.rp2.contains(v); };
    auto add3 = [&](int v) {
        if (s.rp.insert(v)) p.push_back(v);
    };
    auto add2 = [&](int v) {
        p2.push_back(v);
        s.rp2.insert(v);
    };

    if (num <= 4) {
        s.idx.assign(num, 0);
        s.best.assign(num, 0);
        // every access point decoded once: (x, y, layer) by pin and choice
        const int64_t a0 = d.ap_off[pb];
        const int A = (int)(d.ap_off[pb + num] - a0);
        s.ax.resize(A); s.ay.resize(A); s.al.resize(A); s.aoff.resize(num);
        for (int i = 0; i < num; i++) s.aoff[i] = (int)(d.ap_off[pb + i] - a0);
        for (int a = 0; a < A; a++) {
            const int v = d.ap[a0 + a];
            s.ax[a] = v / Y % X; s.ay[a] = v % Y; s.al[a] = v / XY;
        }
        const int *ax = s.ax.data(), *ay = s.ay.data(), *al = s.al.data(), *ao = s.aoff.data();
        int min_diff = 1000000000, min_m = 1000000000, min_m2 = 1000000000, min_m0 = 1000000000;
        // odometer over access-point choices, pin 0 most significant
        while (true) {
            int xmn = 1000000000, xmx = 0, ymn = 1000000000, ymx = 0, diff = 0, m = 0, m2 = 0;
            for (int i = 0; i < num; i++) {
                const int a = ao[i] + s.idx[i];
                const int xi = ax[a], yi = ay[a], li = al[a];
                xmn = std::min(xmn, xi); xmx = std::max(xmx, xi);
                ymn = std::min(ymn, yi); ymx = std::max(ymx, yi);
                m += std::abs(2 * xi - c2x) + std::abs(2 * yi - c2y);
                m2 += li;
                for (int j = 0; j < i; j++) {
                    const int b = ao[j] + s.idx[j];
                    diff += (xi != ax[b]) + (yi != ay[b]);
                }
            }
            int m0 = xmx - xmn + ymx - ymn;
            if (diff < min_diff || (diff == min_diff && m0 < min_m0)) {
                s.best = s.idx; min_diff = diff; min_m0 = m0; min_m = m; min_m2 = m2;
            } else if (diff == min_diff && m0 == min_m0 && m < min_m) {
                s.best = s.idx; min_diff = diff; min_m = m; min_m2 = m2;
            } else if (diff == min_diff && m0 == min_m0 && m == min_m && m2 < min_m2) {
                s.best = s.idx; min_m2 = m2;
            }
            int k = num - 1;
            while (k >= 0 && s.idx[k] + 1 == nap(k)) s.idx[k--] = 0;
            if (k < 0) break;
            s.idx[k]++;
        }
        for (int i = 0; i < num; i++) {
            int v = apv(i, s.best[i]);
            add3(v);
            if (!has2(v % XY)) add2(v % XY);
        }
    } else {
        s.visited.assign(num, 0);
        s.xcnt.next(X);
        s.ycnt.next(Y);
        const int64_t a0 = d.ap_off[pb];
        const int A = (int)(d.ap_off[pb + num] - a0);
        // walk order (src/database.hpp:101-117): the 2-D keys of all access
        // points enter a robin_hood map in first-seen order, each with the pins
        // that have an access point there (ascending); the pins of every key, in
        // the map's iteration order, fill a robin_hood set, whose iteration order
        // every round then follows
        s.keys2d.reset();
        s.first2d.clear();
        s.rank.reset((size_t)A);
        s.ap_rank.resize(A);
        for (int i = 0; i < num; i++)
            for (int j = 0; j < nap(i); j++) {
                const int q = apv(i, j) % XY;
                const int r = s.rank.find_or_insert(q, (int)s.first2d.size());
                if (r == (int)s.first2d.size()) {
                    s.first2d.push_back(q);
                    s.keys2d.insert(q);
                }
                s.ap_rank[d.ap_off[pb + i] - a0 + j] = r;
            }
        const int K = (int)s.first2d.size();
        // pins per 2-D key in push order (i ascending, then j): a counting sort
        s.list_off.assign(K + 1, 0);
        for (int a = 0; a < A; a++) s.list_off[s.ap_rank[a] + 1]++;
        for (int r = 0; r < K; r++) s.list_off[r + 1] += s.list_off[r];
        s.list_pin.resize(A);
        {
            std::vector<int> &fill = s.cnt;  // write cursors
            fill.assign(s.list_off.begin(), s.list_off.end() - 1);
            for (int i = 0; i < num; i++)
                for (int j = 0; j < nap(i); j++) s.list_pin[fill[s.ap_rank[d.ap_off[pb + i] - a0 + j]]++] = i;
        }
        s.walk.reset();
        s.keys2d.for_each([&](int q) {
            const int r = s.rank.find(q);
            for (int t = s.list_off[r]; t < s.list_off[r + 1]; t++) s.walk.insert(s.list_pin[t]);
        });
        s.order.clear();
        s.walk.for_each([&](int i) { s.order.push_back(i); });
        s.cnt.assign(K, 0);
        s.cnt_st.assign(K, 0);
        s.round_st = 0;
        s.kx.resize(K); s.ky.resize(K); s.kd.resize(K);
        for (int r = 0; r < K; r++) {
            const int q = s.first2d[r];
            s.kx[r] = q / Y;
            s.ky[r] = q % Y;
            s.kd[r] = std::abs(s.kx[r] * 2 - c2x) + std::abs(s.ky[r] * 2 - c2y);
        }
        for (int round = 0; round < num; round++) {
            int max_pos = -1, max_rank = -1, cnt_repeat = 0, max_coord = -1, min_dist = 1000000000;
            ++s.round_st;  // every key's running count starts at zero
            for (int i : s.order) {
                if (s.visited[i]) continue;
                const int *rk = s.ap_rank.data() + (d.ap_off[pb + i] - a0);
                for (int j = 0; j < nap(i); j++) {
                    const int r = rk[j], q = s.first2d[r];
                    if (s.cnt_st[r] != s.round_st) {
                        s.cnt_st[r] = s.round_st;
                        s.cnt[r] = 0;
                    }
                    const int sz = ++s.cnt[r];
                    const int dist = s.kd[r];
                    const int coord = s.xcnt.get(s.kx[r]) + s.ycnt.get(s.ky[r]);
                    if (sz > cnt_repeat) {
                        max_pos = q; max_rank = r; cnt_repeat = sz; max_coord = coord; min_dist = dist;
                    } else if (sz == cnt_repeat && coord > max_coord) {
                        max_pos = q; max_rank = r; max_coord = coord; min_dist = dist;
                    } else if (sz == cnt_repeat && coord == max_coord && dist < min_dist) {
                        max_pos = q; max_rank = r; min_dist = dist;
                    }
                }
            }
            if (cnt_repeat <= 1) break;
            if (!has2(max_pos)) {
                add2(max_pos);
                s.xcnt.inc(max_pos / Y % X);
                s.ycnt.inc(max_pos % Y);
            }
            // the pins that had an access point at max_pos this round, in the
            // order of the walk (a pin twice when two of its points are there)
            s.lst.clear();
            for (int i : s.order) {
                if (s.visited[i]) continue;
                const int *rk = s.ap_rank.data() + (d.ap_off[pb + i] - a0);
                for (int j = 0; j < nap(i); j++)
                    if (rk[j] == max_rank) s.lst.push_back(i);
            }
            for (int pin : s.lst) {
                if (s.visited[pin]) throw Error(ERR_FORMAT, "a pin has two access points on one 2-D position");
                s.visited[pin] = 1;
                for (int j = 0; j < nap(pin); j++)
                    if (apv(pin, j) % XY == max_pos) {
                        add3(apv(pin, j));
                        break;
                    }
            }
        }
        for (int i = 0; i < num; i++) {
            if (s.visited[i]) continue;
            int min_dist = 1000000000, chosen = -1, max_overlap = 0;
            for (int j = 0; j < nap(i); j++) {
                int v = apv(i, j), q = v % XY;
                int dist = std::abs(v / Y % X * 2 - c2x) + std::abs(v % Y * 2 - c2y);
                int coord = s.xcnt.get(q / Y) + s.ycnt.get(q % Y);
                if (coord > max_overlap) { max_overlap = coord; min_dist = dist; chosen = v; }
                else if (coord == max_overlap && dist < min_dist) { min_dist = dist; chosen = v; }
            }
            if (chosen < 0) throw Error(ERR_FORMAT, "pin without access points");
            add3(chosen);
            if (!has2(chosen % XY)) {
                add2(chosen % XY);
                s.xcnt.inc(chosen / Y % X);
                s.ycnt.inc(chosen % Y);
            }
        }
        if (p2.size() < p.size()) {
            // stacked pins: per 2-D key the lowest and highest chosen position
            s.mn.assign(K, -1);
            s.mx.assign(K, -1);
            for (int v : p) {
                const int r = s.rank.find(v % XY);
                if (s.mn[r] < 0 || v < s.mn[r]) s.mn[r] = v;
                if (s.mx[r] < 0 || v > s.mx[r]) s.mx[r] = v;
            }
            s.rp2.for_each([&](int q) {
                const int r = s.rank.find(q);
                pins.push_back(s.mx[r]);
                if (s.mn[r] != s.mx[r]) { extra.push_back(s.mn[r]); extra.push_back(s.mx[r]); }
            });
        } else {
            s.rp.for_each([&](int v) { pins.push_back(v); });
        }
        return;
    }
    // output in the iteration order of the reference's sets (src/database.hpp:225-242)
    if (p2.size() < p.size()) {
        s.rp2.for_each([&](int q) {
            int mn = -1, mx = -1;
            for (int v : p)
                if (v % XY == q) {
                    if (mn < 0 || v < mn) mn = v;
                    if (mx < 0 || v > mx) mx = v;
                }
            pins.push_back(mx);
            if (mn != mx) { extra.push_back(mn); extra.push_back(mx); }
        });
    } else {
        s.rp.for_each([&](int v) { pins.push_back(v); });
    }
}

}  // namespace

void select_pins(Design &d, int threads) {
    const int N = d.num_nets();
    if (threads <= 0) threads = hw_threads();
    // ranges of nets, many per thread and handed out dynamically: a few nets
    // of hundreds of pins cost as much as thousands of two-pin nets
    int T = std::max(1, std::min(threads * 32, N / 256 + 1));
    std::vector<std::vector<int>> pins(T), extra(T);
    std::vector<std::vector<int64_t>> pcount(T), ecount(T);
    std::vector<int> lo(T + 1);
    for (int t = 0; t <= T; t++) lo[t] = (int)((int64_t)N * t / T);
    parallel_for(T, threads, [&](int b, int e) {
        PinScratch s;
        for (int t = b; t < e; t++)
            for (int n = lo[t]; n < lo[t + 1]; n++) {
                size_t p0 = pins[t].size(), e0 = extra[t].size();
                select_one(d, n, s, pins[t], extra[t]);
                pcount[t].push_back((int64_t)(pins[t].size() - p0));
                ecount[t].push_back((int64_t)(extra[t].size() - e0));
            }
    });
    // the ranges' selections go to their places in the design's arrays in
    // parallel (and their buffers are freed there), at the prefix sums of
    // the ranges' sizes
    std::vector<int64_t> pb(T + 1, 0), eb(T + 1, 0);
    for (int t = 0; t < T; t++) {
        pb[t + 1] = pb[t] + (int64_t)pins[t].size();
        eb[t + 1] = eb[t] + (int64_t)extra[t].size();
    }
    d.sel_off.assign(N + 1, 0); d.extra_off.assign(N + 1, 0);
    d.sel.resize(pb[T]); d.extra.resize(eb[T]);
    parallel_for(T, threads, [&](int b, int e) {
        for (int t = b; t < e; t++) {
            std::copy(pins[t].begin(), pins[t].end(), d.sel.begin() + pb[t]);
            std::copy(extra[t].begin(), extra[t].end(), d.extra.begin() + eb[t]);
            int64_t ps = pb[t], es = eb[t];
            for (int n = lo[t]; n < lo[t + 1]; n++) {
                ps += pcount[t][n - lo[t]];
                es += ecount[t][n - lo[t]];
                d.sel_off[n + 1] = ps;
                d.extra_off[n + 1] = es;
            }
            std::vector<int>().swap(pins[t]);
            std::vector<int>().swap(extra[t]);
        }
    });
}

}  // namespace igr
