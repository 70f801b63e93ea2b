// Deterministic rectilinear Steiner tree provider.
//
// InstantGR builds its trees with FLUTE (src/flute.hpp), whose topology table
// POST9.dat is not shipped with it (it is listed in .MISSING_LARGE_BLOBS), so
// upstream FLUTE cannot run for degree >= 4.  This provider takes its place on
// both sides of every comparison: the router of this project links it, and the
// reference build used for baselines links it through a flute.hpp stand-in.
//
// Method (all in the caller's coordinate space, i.e. DR units):
//   1. distinct points, sorted by (x, y);
//   2. rectilinear minimum spanning tree by Kruskal over candidate edges: all
//      pairs up to 64 points, otherwise the four-octant sweep of Zhou, Shenoy
//      and Nicholls ("Efficient minimum spanning tree construction without
//      Delaunay triangulation", 2002), edges ordered by (length, lo, hi);
//   3. Steinerisation: for every node and every pair of its tree neighbours the
//      median point of the three is tried; the best strictly positive saving
//      is applied (edges v-a, v-b replaced by s-v, s-a, s-b), repeated for up
//      to four passes; Steiner points of degree <= 2 are then spliced out.
//      Degree three is FLUTE's closed form: the median point of the three.
// The result does not depend on the order of the input points.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <climits>
#include <stdexcept>
#include <numeric>
#include <utility>
#include <vector>

namespace igr_steiner {

struct Tree {
    std::vector<int> x, y;                   // node coordinates: pins first, then Steiner points
    std::vector<std::pair<int, int>> edges;  // undirected tree edges
    int npins = 0;
};

inline int med3(int a, int b, int c) { return std::max(std::min(a, b), std::min(std::max(a, b), c)); }

// Sorts 64-bit keys ascending: a least-significant-digit radix sort over the
// bytes in which the keys differ (std::sort for few keys).  Any correct sort
// gives the same sequence of keys, so the trees do not depend on which one
// runs.
inline void sort_keys(std::vector<uint64_t> &a, std::vector<uint64_t> &tmp) {
    const size_t n = a.size();
    if (n < 256) {
        std::sort(a.begin(), a.end());
        return;
    }
    uint64_t all_or = 0, all_and = ~0ull;
    for (uint64_t k : a) { all_or |= k; all_and &= k; }
    const uint64_t differ = all_or ^ all_and;
    tmp.resize(n);
    for (int shift = 0; shift < 64; shift += 8) {
        if (((differ >> shift) & 0xff) == 0) continue;
        size_t cnt[257] = {};
        for (uint64_t k : a) cnt[((k >> shift) & 0xff) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (uint64_t k : a) tmp[cnt[(k >> shift) & 0xff]++] = k;
        a.swap(tmp);
    }
}

// The node at each position of a large tree: open addressing with linear
// probing (a lookup answers the same as any map would).
struct PosMap {
    std::vector<int64_t> key;
    std::vector<int> val;
    std::vector<uint8_t> used;
    size_t mask = 0, n = 0;
    static size_t slot(int64_t k) { return (size_t)(((uint64_t)k * 0x9E3779B97F4A7C15ull) >> 24); }
    void reset(size_t expect) {
        size_t cap = 64;
        while (cap < 4 * expect) cap <<= 1;
        key.resize(cap);
        val.resize(cap);
        used.assign(cap, 0);
        mask = cap - 1;
        n = 0;
    }
    void put(int64_t k, int v) {
        if (2 * (n + 1) > mask + 1) grow();
        size_t i = slot(k) & mask;
        while (used[i] && key[i] != k) i = (i + 1) & mask;
        if (!used[i]) { used[i] = 1; key[i] = k; n++; }
        val[i] = v;
    }
    int get(int64_t k) const {
        for (size_t i = slot(k) & mask; used[i]; i = (i + 1) & mask)
            if (key[i] == k) return val[i];
        return -1;
    }
    void grow() {
        std::vector<int64_t> k0;
        std::vector<int> v0;
        std::vector<uint8_t> u0;
        k0.swap(key);
        v0.swap(val);
        u0.swap(used);
        reset(u0.size());
        for (size_t i = 0; i < u0.size(); i++)
            if (u0[i]) put(k0[i], v0[i]);
    }
};

// Containers of one build, kept per thread so that the small trees of most
// nets allocate nothing.
struct BuildScratch {
    std::vector<std::pair<int, int>> pts;
    std::vector<uint64_t> pkey, ktmp;
    std::vector<std::vector<int>> adj;  // only the first `used` lists are live
    size_t used = 0;
    std::vector<int> sn, nid, nx, ny;
    std::vector<long long> key;
    std::vector<int> from, out, touched, clean;
    PosMap at;
    // n empty adjacency lists
    void lists(size_t n) {
        for (size_t v = 0; v < std::min(n, adj.size()); v++) adj[v].clear();
        if (adj.size() < n) adj.resize(n);
        used = n;
    }
    void add_list() {
        if (adj.size() <= used) adj.emplace_back();
        adj[used++].clear();
    }
};

inline BuildScratch &build_scratch() {
    thread_local BuildScratch s;
    return s;
}

inline void build(const std::vector<int> &xin, const std::vector<int> &yin, Tree &t) {
    t.x.clear();
    t.y.clear();
    t.edges.clear();
    t.npins = 0;
    BuildScratch &bs = build_scratch();
    const int n0 = (int)xin.size();
    std::vector<std::pair<int, int>> &pts = bs.pts;
    pts.resize(n0);
    if (n0 < 256) {
        for (int i = 0; i < n0; i++) pts[i] = {xin[i], yin[i]};
        std::sort(pts.begin(), pts.end());
    } else {
        // (x, y) as one key that sorts as the pair does (sign bits flipped)
        std::vector<uint64_t> &pk = bs.pkey;
        pk.resize(n0);
        for (int i = 0; i < n0; i++)
            pk[i] = (uint64_t)((uint32_t)xin[i] ^ 0x80000000u) << 32 | ((uint32_t)yin[i] ^ 0x80000000u);
        sort_keys(pk, bs.ktmp);
        for (int i = 0; i < n0; i++)
            pts[i] = {(int)((uint32_t)(pk[i] >> 32) ^ 0x80000000u), (int)((uint32_t)pk[i] ^ 0x80000000u)};
    }
    pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
    const int P = (int)pts.size();
    for (auto &p : pts) { t.x.push_back(p.first); t.y.push_back(p.second); }
    t.npins = P;
    if (P <= 1) return;
    if (P == 2) { t.edges.push_back({0, 1}); return; }
    auto dist = [&](int a, int b) { return std::abs(t.x[a] - t.x[b]) + std::abs(t.y[a] - t.y[b]); };
    if (P == 3) {
        int sx = med3(t.x[0], t.x[1], t.x[2]), sy = med3(t.y[0], t.y[1], t.y[2]);
        int c = -1;
        for (int i = 0; i < 3; i++) if (t.x[i] == sx && t.y[i] == sy) c = i;
        if (c < 0) { t.x.push_back(sx); t.y.push_back(sy); c = 3; }
        for (int i = 0; i < 3; i++) if (i != c) t.edges.push_back({std::min(i, c), std::max(i, c)});
        return;
    }
    // ---- spanning tree: up to kPrimMax points the minimum spanning tree
    // under the strict edge order (length, lo, hi), by Prim over all pairs;
    // above, Kruskal in that order over the sweep candidates (a minimum
    // spanning tree, which can settle ties of length otherwise).  Nothing
    // below depends on the order of a node's neighbour list.
    bs.lists(P);
    std::vector<std::vector<int>> &adj = bs.adj;
    constexpr int kPrimMax = 64;  // (ids fit the 10 bits of the edge key)
    if (P <= kPrimMax) {
        // Prim: key of the best edge from the tree to each outside point, as
        // (length, lo, hi) in one integer (lengths < 2^31)
        std::vector<long long> &key = bs.key;
        std::vector<int> &from = bs.from, &out = bs.out;
        key.resize(P);
        from.resize(P);
        out.resize(P);
        const int *xs = t.x.data(), *ys = t.y.data();
        auto ek = [&](int a, int b) {
            const int lo = a < b ? a : b, hi = a < b ? b : a;
            const long long w = std::abs(xs[a] - xs[b]) + std::abs(ys[a] - ys[b]);
            return (w << 20) | ((long long)lo << 10) | hi;
        };
        // points still outside the tree, compacted as they join; the scan
        // that lowers their keys also finds the next point to join
        int nout = P - 1, bi = 0;
        for (int i = 1; i < P; i++) {
            key[i] = ek(0, i);
            from[i] = 0;
            out[i - 1] = i;
            if (key[i] < key[out[bi]]) bi = i - 1;
        }
        while (nout > 0) {
            const int best = out[bi];
            out[bi] = out[--nout];
            adj[from[best]].push_back(best);
            adj[best].push_back(from[best]);
            bi = 0;
            long long bk = LLONG_MAX;
            for (int k = 0; k < nout; k++) {
                const int i = out[k];
                const long long q = ek(best, i);
                if (q < key[i]) { key[i] = q; from[i] = best; }
                if (key[i] < bk) { bk = key[i]; bi = k; }
            }
        }
    } else {
        // candidate edges as keys length << 32 | lo << 16 | hi (points < 2^16)
        // or, above that, as (length, lo, hi) triples; both sort in the same order
        const bool packed = P < (1 << 16);
        struct E { int w, a, b; };
        std::vector<E> cand;
        std::vector<uint64_t> ckey;
        auto add = [&](int i, int j) {
            const int lo = std::min(i, j), hi = std::max(i, j), w = dist(i, j);
            if (packed) ckey.push_back((uint64_t)(uint32_t)w << 32 | (uint64_t)lo << 16 | (uint64_t)hi);
            else cand.push_back({w, lo, hi});
        };
        (packed ? (void)ckey.reserve((size_t)8 * P) : cand.reserve((size_t)8 * P));
        std::vector<int> px(t.x), py(t.y), id(P);
        std::vector<uint64_t> order(P), stmp;
        std::vector<std::pair<int, int>> sweep;  // (-y, point), ascending
        sweep.reserve(P);
        for (int k = 0; k < 4; k++) {
            // points by x + y, then by index; sums fit 33 bits, indices 31
            // (the sign bit flipped, so that the keys sort as unsigned)
            for (int i = 0; i < P; i++)
                order[i] = (uint64_t)((((int64_t)px[i] + py[i]) << 31) + i) ^ (1ull << 63);
            sort_keys(order, stmp);
            for (int i = 0; i < P; i++) id[i] = (int)(order[i] & 0x7fffffff);
            sweep.clear();
            for (int i : id) {
                auto lo = std::lower_bound(sweep.begin(), sweep.end(), std::make_pair(-py[i], INT32_MIN));
                auto it = lo;
                for (; it != sweep.end(); ++it) {
                    int j = it->second;
                    int dx = px[i] - px[j], dy = py[i] - py[j];
                    if (dy > dx) break;
                    add(i, j);
                }
                // the keys from lo on are >= -py[i]; an equal key was erased above
                // (dy == 0 <= dx for a point swept earlier), so i goes in at lo
                if (it != lo) {
                    *lo = {-py[i], i};
                    sweep.erase(lo + 1, it);
                } else {
                    sweep.insert(lo, {-py[i], i});
                }
            }
            for (int i = 0; i < P; i++) {
                if (k & 1) px[i] = -px[i];
                else std::swap(px[i], py[i]);
            }
        }
        if (packed) {
            sort_keys(ckey, stmp);
            cand.resize(ckey.size());
            for (size_t q = 0; q < ckey.size(); q++)
                cand[q] = {(int)(ckey[q] >> 32), (int)(ckey[q] >> 16 & 0xffff), (int)(ckey[q] & 0xffff)};
        } else {
            std::sort(cand.begin(), cand.end(), [](const E &l, const E &r) {
                if (l.w != r.w) return l.w < r.w;
                if (l.a != r.a) return l.a < r.a;
                return l.b < r.b;
            });
        }
        std::vector<int> uf(P);
        std::iota(uf.begin(), uf.end(), 0);
        auto find = [&](int v) {
            while (uf[v] != v) v = uf[v] = uf[uf[v]];
            return v;
        };
        int used = 0;
        for (auto &e : cand) {
            int ra = find(e.a), rb = find(e.b);
            if (ra == rb) continue;
            uf[ra] = rb;
            adj[e.a].push_back(e.b);
            adj[e.b].push_back(e.a);
            if (++used == P - 1) break;
        }
    }
    // ---- Steinerisation.  The node at a position: a scan over the nodes for
    // small trees, a hash map above (positions are distinct: the pins are, and
    // a Steiner point is only made where no node is)
    const bool scan = P <= 64;  // (independent of the MST method)
    PosMap &at = bs.at;
    auto key = [](int x, int y) { return ((int64_t)x << 32) ^ (uint32_t)y; };
    if (!scan) {
        at.reset((size_t)2 * P);
        for (int i = 0; i < P; i++) at.put(key(t.x[i], t.y[i]), i);
    }
    auto node_at_pos = [&](int x, int y) {
        if (!scan) return at.get(key(x, y));
        for (int v = 0; v < (int)t.x.size(); v++)
            if (t.x[v] == x && t.y[v] == y) return v;
        return -1;
    };
    auto drop = [&](int u, int v) {
        auto &a = adj[u];
        a.erase(std::find(a.begin(), a.end(), v));
    };
    std::vector<int> &sn = bs.sn;
    // a node evaluated without a saving is skipped until its neighbour list
    // changes: the positions never move, so its best saving stays <= 0
    std::vector<int> &touched = bs.touched, &clean = bs.clean;
    touched.assign(bs.used, 0);
    clean.assign(bs.used, -1);
    int tick = 0;
    auto touch = [&](int v) {
        if ((int)touched.size() <= v) { touched.resize(v + 1, 0); clean.resize(v + 1, -1); }
        touched[v] = ++tick;
    };
    for (int pass = 0; pass < 4; pass++) {
        bool changed = false;
        for (int v = 0; v < (int)bs.used; v++) {
            auto &nb = adj[v];
            if (nb.size() < 2) continue;
            if (clean[v] >= touched[v]) continue;
            sn.assign(nb.begin(), nb.end());
            std::sort(sn.begin(), sn.end());
            int best_gain = 0, ba = -1, bb = -1, bx = 0, by = 0;
            for (size_t i = 0; i < sn.size(); i++)
                for (size_t j = i + 1; j < sn.size(); j++) {
                    int a = sn[i], b = sn[j];
                    int sx = med3(t.x[v], t.x[a], t.x[b]), sy = med3(t.y[v], t.y[a], t.y[b]);
                    int g = dist(v, a) + dist(v, b) -
                            (std::abs(sx - t.x[v]) + std::abs(sy - t.y[v]) + std::abs(sx - t.x[a]) +
                             std::abs(sy - t.y[a]) + std::abs(sx - t.x[b]) + std::abs(sy - t.y[b]));
                    if (g > best_gain) { best_gain = g; ba = a; bb = b; bx = sx; by = sy; }
                }
            if (best_gain <= 0) {
                clean[v] = tick;
                continue;
            }
            int s = node_at_pos(bx, by);
            if (s >= 0) {
                if (s != ba && s != bb) continue;  // would merge with an unrelated node
                // s coincides with a neighbour: reattach the other neighbour to it
                int o = (s == ba) ? bb : ba;
                drop(v, o); drop(o, v);
                adj[s].push_back(o); adj[o].push_back(s);
                touch(v); touch(o); touch(s);
            } else {
                s = (int)t.x.size();
                t.x.push_back(bx); t.y.push_back(by);
                bs.add_list();
                if (!scan) at.put(key(bx, by), s);
                drop(v, ba); drop(ba, v); drop(v, bb); drop(bb, v);
                for (int w : {v, ba, bb}) { adj[s].push_back(w); adj[w].push_back(s); }
                touch(v); touch(ba); touch(bb); touch(s);
            }
            changed = true;
        }
        if (!changed) break;
    }
    // splice out Steiner points of degree <= 2
    bool again = true;
    while (again) {
        again = false;
        for (int s = P; s < (int)bs.used; s++) {
            if (adj[s].size() == 1) {
                int a = adj[s][0];
                drop(a, s); adj[s].clear(); again = true;
            } else if (adj[s].size() == 2) {
                int a = adj[s][0], b = adj[s][1];
                drop(a, s); drop(b, s); adj[s].clear();
                adj[a].push_back(b); adj[b].push_back(a);
                again = true;
            }
        }
    }
    // compact node ids (drop emptied Steiner points)
    const int V = (int)bs.used;
    std::vector<int> &nid = bs.nid;
    nid.assign(V, -1);
    int k = 0;
    for (int v = 0; v < V; v++)
        if (v < P || !adj[v].empty()) nid[v] = k++;
    std::vector<int> &nx = bs.nx, &ny = bs.ny;
    nx.resize(k);
    ny.resize(k);
    for (int v = 0; v < V; v++)
        if (nid[v] >= 0) { nx[nid[v]] = t.x[v]; ny[nid[v]] = t.y[v]; }
    for (int v = 0; v < V; v++)
        for (int w : adj[v])
            if (v < w) t.edges.push_back({nid[v], nid[w]});
    if (t.edges.size() < 256) {
        std::sort(t.edges.begin(), t.edges.end());
    } else {  // node ids are >= 0: (a, b) as one key
        std::vector<uint64_t> &ek2 = bs.pkey;
        ek2.resize(t.edges.size());
        for (size_t i = 0; i < t.edges.size(); i++)
            ek2[i] = (uint64_t)(uint32_t)t.edges[i].first << 32 | (uint32_t)t.edges[i].second;
        sort_keys(ek2, bs.ktmp);
        for (size_t i = 0; i < t.edges.size(); i++) t.edges[i] = {(int)(ek2[i] >> 32), (int)(uint32_t)ek2[i]};
    }
    t.x.assign(nx.begin(), nx.end());
    t.y.assign(ny.begin(), ny.end());
}

// FLUTE-style branch list for d input points (d >= 2): 2d-2 branches, branch i
// < d is input point i, branches d.. are Steiner points, branch.n is the
// neighbour towards the root (node 0), the root points at itself, and unused
// slots repeat the root.  This is the contract of flute::Tree
// (src/flute.hpp:43-56) consumed by the reference's my_flute
// (src/database_cuda.hpp:696-744).
struct Branch { int x, y, n; };
inline void to_branches(const std::vector<int> &xin, const std::vector<int> &yin, const Tree &t,
                        std::vector<Branch> &br) {
    const int d = (int)xin.size();
    br.assign(std::max(0, 2 * d - 2), Branch{0, 0, 0});
    if (d < 2) return;
    const int V = (int)t.x.size();
    struct Scratch {
        std::vector<std::vector<int>> adj;
        std::vector<int> par, order, bidx, node_of;
    };
    thread_local Scratch ts;
    std::vector<std::vector<int>> &adj = ts.adj;
    if ((int)adj.size() < V) adj.resize(V);
    for (int v = 0; v < V; v++) adj[v].clear();
    for (auto &e : t.edges) { adj[e.first].push_back(e.second); adj[e.second].push_back(e.first); }
    std::vector<int> &par = ts.par, &order = ts.order;
    par.assign(V, -1);
    order.clear();
    order.push_back(0);
    par[0] = 0;
    for (size_t i = 0; i < order.size(); i++)
        for (int w : adj[order[i]])
            if (par[w] < 0) { par[w] = order[i]; order.push_back(w); }
    // branch index of each tree node: first input point at that position, or a Steiner slot
    std::vector<int> &bidx = ts.bidx;
    bidx.assign(V, -1);
    // tree node of each input point: the pins come first in (x, y) order, distinct
    auto node_at = [&](int x, int y) {
        int lo = 0, hi = t.npins;
        while (lo < hi) {
            const int m = (lo + hi) >> 1;
            if (t.x[m] < x || (t.x[m] == x && t.y[m] < y)) lo = m + 1;
            else hi = m;
        }
        if (lo == t.npins || t.x[lo] != x || t.y[lo] != y) throw std::out_of_range("point not in the tree");
        return lo;
    };
    std::vector<int> &node_of = ts.node_of;
    node_of.resize(d);
    for (int i = 0; i < d; i++) {
        const int v = node_of[i] = node_at(xin[i], yin[i]);
        if (bidx[v] < 0) bidx[v] = i;
    }
    int slot = d;
    for (int v = t.npins; v < V; v++) bidx[v] = slot++;
    for (int v = 0; v < V; v++) br[bidx[v]] = Branch{t.x[v], t.y[v], bidx[par[v]]};
    for (int i = 0; i < d; i++) {
        const int v = node_of[i];
        if (bidx[v] != i) br[i] = Branch{xin[i], yin[i], bidx[v]};  // duplicate input point
    }
    for (int s = slot; s < 2 * d - 2; s++) br[s] = Branch{t.x[0], t.y[0], bidx[0]};
}

}  // namespace igr_steiner
