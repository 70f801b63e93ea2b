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
#include <unordered_map>

namespace igr {

namespace {

struct PinScratch {
    std::vector<int> idx, best;
    std::unordered_map<int, std::vector<int>> cnt2d;
    std::unordered_map<int, int> xcnt, ycnt;
    std::vector<char> visited;
    std::vector<int> p, p2;
    std::vector<int> order;        // walk order of the pins in the greedy rounds
    RobinOrder keys2d, walk, rp, rp2;
    std::vector<int> first2d;            // 2-D keys in first-seen order; pins per key (CSR below)
    std::vector<int> list_off, list_pin;
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
    auto has2 = [&](int v) { return std::find(p2.begin(), p2.end(), v) != p2.end(); };
    // the reference's robin_hood sets p and p2D (their insertion sequences)
    auto add3 = [&](int v) {
        if (std::find(p.begin(), p.end(), v) == p.end()) p.push_back(v);
        s.rp.insert(v);
    };
    auto add2 = [&](int v) {
        p2.push_back(v);
        s.rp2.insert(v);
    };

    if (num <= 4) {
        s.idx.assign(num, 0);
        s.best.assign(num, 0);
        int min_diff = 1000000000, min_m = 1000000000, min_m2 = 1000000000, min_m0 = 1000000000;
        // odometer over access-point choices, pin 0 most significant
        while (true) {
            int xmn = 1000000000, xmx = 0, ymn = 1000000000, ymx = 0, diff = 0, m = 0, m2 = 0;
            for (int i = 0; i < num; i++) {
                int v = apv(i, s.idx[i]);
                int xi = v / Y % X, yi = v % Y, li = v / XY;
                xmn = std::min(xmn, xi); xmx = std::max(xmx, xi);
                ymn = std::min(ymn, yi); ymx = std::max(ymx, yi);
                m += std::abs(2 * xi - c2x) + std::abs(2 * yi - c2y);
                m2 += li;
                for (int j = 0; j < i; j++) {
                    int w = apv(j, s.idx[j]);
                    diff += (xi != w / Y % X) + (yi != w % Y);
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
        s.xcnt.clear(); s.ycnt.clear();
        auto cnt_of = [](std::unordered_map<int, int> &m, int k) {
            auto it = m.find(k);
            return it == m.end() ? 0 : it->second;
        };
        // walk order (src/database.hpp:101-117): the 2-D keys of all access
        // points enter a robin_hood map in first-seen order, each with the pins
        // that have an access point there (ascending); the pins of every key, in
        // the map's iteration order, fill a robin_hood set, whose iteration order
        // every round then follows
        s.keys2d.reset();
        s.first2d.clear();
        for (int i = 0; i < num; i++)
            for (int j = 0; j < nap(i); j++) {
                const int q = apv(i, j) % XY;
                if (s.keys2d.insert(q)) s.first2d.push_back(q);
            }
        {
            // pins per 2-D key, in push order (i ascending, then j)
            std::vector<std::pair<int, int>> kp;  // (key rank in first2d, pin)
            std::unordered_map<int, int> rank;
            for (size_t r = 0; r < s.first2d.size(); r++) rank[s.first2d[r]] = (int)r;
            for (int i = 0; i < num; i++)
                for (int j = 0; j < nap(i); j++) kp.push_back({rank[apv(i, j) % XY], i});
            std::stable_sort(kp.begin(), kp.end(),
                             [](const std::pair<int, int> &a, const std::pair<int, int> &b) { return a.first < b.first; });
            s.list_off.assign(s.first2d.size() + 1, 0);
            s.list_pin.clear();
            for (auto &e : kp) {
                s.list_off[e.first + 1]++;
                s.list_pin.push_back(e.second);
            }
            for (size_t r = 0; r < s.first2d.size(); r++) s.list_off[r + 1] += s.list_off[r];
            s.walk.reset();
            s.keys2d.for_each([&](int q) {
                const int r = rank[q];
                for (int t = s.list_off[r]; t < s.list_off[r + 1]; t++) s.walk.insert(s.list_pin[t]);
            });
            s.order.clear();
            s.walk.for_each([&](int i) { s.order.push_back(i); });
        }
        for (int round = 0; round < num; round++) {
            int max_pos = -1, cnt_repeat = 0, max_coord = -1, min_dist = 1000000000;
            s.cnt2d.clear();
            for (int i : s.order) {
                if (s.visited[i]) continue;
                for (int j = 0; j < nap(i); j++) {
                    int q = apv(i, j) % XY;
                    auto &lst = s.cnt2d[q];
                    lst.push_back(i);
                    int dist = std::abs(q / Y * 2 - c2x) + std::abs(q % Y * 2 - c2y);
                    int coord = cnt_of(s.xcnt, q / Y) + cnt_of(s.ycnt, q % Y);
                    int sz = (int)lst.size();
                    if (sz > cnt_repeat) {
                        max_pos = q; cnt_repeat = sz; max_coord = coord; min_dist = dist;
                    } else if (sz == cnt_repeat && coord > max_coord) {
                        max_pos = q; max_coord = coord; min_dist = dist;
                    } else if (sz == cnt_repeat && coord == max_coord && dist < min_dist) {
                        max_pos = q; min_dist = dist;
                    }
                }
            }
            if (cnt_repeat <= 1) break;
            if (!has2(max_pos)) {
                add2(max_pos);
                s.xcnt[max_pos / Y % X]++;
                s.ycnt[max_pos % Y]++;
            }
            for (int pin : s.cnt2d[max_pos]) {
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
                int coord = cnt_of(s.xcnt, q / Y) + cnt_of(s.ycnt, q % Y);
                if (coord > max_overlap) { max_overlap = coord; min_dist = dist; chosen = v; }
                else if (coord == max_overlap && dist < min_dist) { min_dist = dist; chosen = v; }
            }
            if (chosen < 0) throw Error(ERR_FORMAT, "pin without access points");
            add3(chosen);
            if (!has2(chosen % XY)) {
                add2(chosen % XY);
                s.xcnt[chosen / Y % X]++;
                s.ycnt[chosen % Y]++;
            }
        }
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
    int T = std::max(1, std::min(threads, N / 256 + 1));
    std::vector<std::vector<int>> pins(T), extra(T);
    std::vector<std::vector<int64_t>> pcount(T), ecount(T);
    std::vector<int> lo(T + 1);
    for (int t = 0; t <= T; t++) lo[t] = (int)((int64_t)N * t / T);
    parallel_for(T, T, [&](int b, int e) {
        PinScratch s;
        for (int t = b; t < e; t++)
            for (int n = lo[t]; n < lo[t + 1]; n++) {
                size_t p0 = pins[t].size(), e0 = extra[t].size();
                select_one(d, n, s, pins[t], extra[t]);
                pcount[t].push_back((int64_t)(pins[t].size() - p0));
                ecount[t].push_back((int64_t)(extra[t].size() - e0));
            }
    });
    d.sel_off.assign(1, 0); d.extra_off.assign(1, 0);
    d.sel.clear(); d.extra.clear();
    d.sel_off.reserve(N + 1); d.extra_off.reserve(N + 1);
    for (int t = 0; t < T; t++) {
        for (auto c : pcount[t]) d.sel_off.push_back(d.sel_off.back() + c);
        for (auto c : ecount[t]) d.extra_off.push_back(d.extra_off.back() + c);
        d.sel.insert(d.sel.end(), pins[t].begin(), pins[t].end());
        d.extra.insert(d.extra.end(), extra[t].begin(), extra[t].end());
    }
}

}  // namespace igr
