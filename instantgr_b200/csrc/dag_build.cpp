// Detour DAG of one net for phase 2 (rip-up and reroute).
//
// Restates net::generate_detours_reconstruct (src/database_cuda.hpp:1429-2086)
// with construct_segments = false, in this project's own code:
//   1. root = last node popped by a leaf-peeling BFS (select_root_net, :826-856);
//   2. congestion regions per direction: a DFS from the root groups tree
//      nodes joined by congested straight edges (union-find with path
//      compression), collecting "stems" (pin coordinates across the trunk) and
//      the trunk's extent (:1494-1637);
//   3. a DFS over the tree creates DAG nodes: each tree node, mirrored copies
//      of congested trunks shifted to positions chosen by the stem
//      displacement rule (get_mirror_places, :1734-1772), both L-shapes and the
//      best `select` Z-shapes of every bent edge ranked by the congestion
//      prefix sums, and long edges split at 50/150 GCells (connect_node,
//      :1671-1724); every connection records (parent, child slot);
//   4. nodes are renumbered so that parents precede children and each node's
//      depth is its longest distance from the root (:2027-2085).
// The quirks of the reference are kept because they shape the DAG: the
// upward probe of the mirror range tests position high-1 (:1750), Z-shape
// candidates that were never scored keep the value-initialised (0, 0) slot
// of std::pair and are then skipped by the bounds checks, and congestion of a
// horizontal Z leg is read from the y prefix sums (:1885-1887).
#include "host.hpp"

#include <algorithm>
#include <queue>
#include <stack>

namespace igr {

namespace {

// Working arrays of one builder, kept per host thread so that their capacity
// carries over from net to net.
struct Scratch {
    std::vector<int> region[2];
    std::vector<std::pair<int, int>> range[2];
    std::vector<std::vector<int>> stems[2];
    std::vector<int> nodes, child_pre, points;
    std::vector<std::pair<int, int>> links;
    std::vector<int> poff, pcode, at, visit, newid, stk;
    std::vector<std::pair<int, int>> st;
};

struct Builder {
    const NetSet &ns;
    const RNet &net;
    const CongestionView &cv;
    int mode;
    DagNet &out;
    int X, Y, XY;
    const TreeAdj &G;                        // tree adjacency
    const std::pmr::vector<int> &P;          // tree node positions (3-D, Steiner layer 9)
    int ntree;
    float ratio;
    int num_tracks;
    int root = -1;
    Scratch &sc;
    std::vector<int> (&region)[2];
    std::vector<std::pair<int, int>> (&range)[2];
    std::vector<std::vector<int>> (&stems)[2];
    // DAG under construction
    std::vector<int> &nodes;
    std::vector<std::pair<int, int>> &links;  // (child, parent*10 + slot) in creation order
    std::vector<int> &child_pre;
    std::vector<int> &points;

    Builder(const NetSet &n_, const RNet &r, const CongestionView &c, int m, DagNet &o, Scratch &s)
        : ns(n_), net(r), cv(c), mode(m), out(o), X(n_.X), Y(n_.Y), XY(n_.X * n_.Y), G(r.adj), P(r.tnode),
          ntree((int)r.tnode.size()), sc(s), region(s.region), range(s.range), stems(s.stems), nodes(s.nodes),
          links(s.links), child_pre(s.child_pre), points(s.points) {
        ratio = 0.15f;
        num_tracks = 9;
        if (mode == 0 || mode == 1) { ratio = 0.1f; num_tracks = 6; }
        nodes.clear();
        links.clear();
        child_pre.clear();
        points.clear();
    }

    int px_(int v) const { return v / Y % X; }
    int py_(int v) const { return v % Y; }
    float ys(int x, int y) const { return cv.ysum[(size_t)x * Y + y]; }
    float xs(int x, int y) const { return cv.xsum[(size_t)x * Y + y]; }

    int select_root() {
        std::queue<std::pair<int, int>> q;
        std::vector<char> vis(ntree, 0);
        int sel = -1;
        for (int i = 0; i < ntree; i++)
            if (G[i].size() == 1) q.push({i, -1});
        while (!q.empty()) {
            auto f = q.front();
            q.pop();
            sel = f.first;
            if (vis[sel]) continue;
            vis[sel] = 1;
            for (int j : G[sel])
                if (j != f.second) q.push({j, sel});
        }
        return sel;
    }

    int region_of(int x, int dir) {
        if (x == -1) return -1;
        if (region[dir][x] == -1) return -1;
        if (region[dir][x] != x) {
            int a = region_of(region[dir][x], dir);
            region[dir][x] = a;
            return a;
        }
        return x;
    }

    void mark(int x, int par) {
        const int cx = px_(P[x]), cy = py_(P[x]);
        for (int e : G[x]) {
            if (e == par) continue;
            const int ex = px_(P[e]), ey = py_(P[e]);
            int dir = -1, cong = -1;
            if (ex == cx) {
                if (ys(cx, std::max(ey, cy)) - ys(cx, std::min(ey, cy)) > 0) { dir = 1; cong = 1; }
            } else if (ey == cy) {
                if (xs(std::max(ex, cx), cy) - xs(std::min(ex, cx), cy) > 0) { dir = 0; cong = 1; }
            } else {
                bool cyy = (ys(cx, std::max(ey, cy)) - ys(cx, std::min(ey, cy))) > 0 ||
                           (ys(ex, std::max(ey, cy)) - ys(ex, std::min(ey, cy))) > 0;
                if (cyy) { dir = 1; cong = 2; }
                if (cong == -1) {
                    bool cxx = (xs(std::max(ex, cx), cy) - xs(std::min(ex, cx), cy)) > 0 ||
                               (xs(std::max(ex, cx), ey) - xs(std::min(ex, cx), ey)) > 0;
                    if (cxx) { dir = 0; cong = 2; }
                }
            }
            if (cong == 1) {
                int target;
                if (x != root) {
                    if (region[dir][x] == -1) region[dir][x] = x;
                    target = region_of(x, dir);
                } else {
                    if (region[dir][e] == -1) region[dir][e] = e;
                    target = region_of(e, dir);
                }
                region[dir][e] = target;
                if (x != root) {
                    std::vector<int> add(stems[dir][e]);
                    stems[dir][target].insert(stems[dir][target].end(), add.begin(), add.end());
                }
                range[dir][target].first = std::min(range[dir][target].first, range[dir][e].first);
                range[dir][target].second = std::max(range[dir][target].second, range[dir][e].second);
            } else if (cong == 2) {
                if (x != root && region[dir][x] == -1) region[dir][x] = x;
                if (region[dir][e] == -1) region[dir][e] = e;
            }
            mark(e, x);
        }
        for (int dir = 0; dir < 2; dir++) {
            const int xr = region_of(x, dir);
            for (int e : G[x]) {
                if (e == par) continue;
                const int ex = px_(P[e]), ey = py_(P[e]);
                const int er = region_of(e, dir);
                if (xr != er) {
                    if (xr >= 0) {
                        stems[dir][xr].push_back(dir ? ex : ey);
                        range[dir][xr].first = std::min(range[dir][xr].first, dir ? ey : ex);
                        range[dir][xr].second = std::max(range[dir][xr].second, dir ? ey : ex);
                    }
                    if (er >= 0) {
                        stems[dir][er].push_back(dir ? cx : cy);
                        range[dir][er].first = std::min(range[dir][er].first, dir ? cy : cx);
                        range[dir][er].second = std::max(range[dir][er].second, dir ? cy : cx);
                    }
                }
            }
        }
    }

    int create(int l, int x, int y) {
        nodes.push_back(l * XY + x * Y + y);
        child_pre.push_back(0);
        return (int)nodes.size() - 1;
    }

    void connect_pre(int p, int c, int slot) {
        points.push_back(px_(nodes[c]) * Y + py_(nodes[c]));
        points.push_back(px_(nodes[p]) * Y + py_(nodes[p]));
        links.push_back({c, p * 10 + slot});
        child_pre[p]++;
    }

    void connect(int p, int c, int slot) {
        const int ax = px_(nodes[p]), ay = py_(nodes[p]), bx = px_(nodes[c]), by = py_(nodes[c]);
        const int len = std::abs(ax - bx) + std::abs(ay - by);
        if (len < 50) { connect_pre(p, c, slot); return; }
        if (len < 150) {
            int m = create(9, (ax + bx) / 2, (ay + by) / 2);
            connect_pre(p, m, slot);
            connect_pre(m, c, 0);
            return;
        }
        int m1, m2;
        if (ay == by) {
            m1 = create(9, ax * 2 / 3 + bx / 3, ay);
            m2 = create(9, ax * 1 / 3 + bx * 2 / 3, ay);
        } else if (ax == bx) {
            m1 = create(9, ax, ay * 2 / 3 + by / 3);
            m2 = create(9, ax, ay * 1 / 3 + by * 2 / 3);
        } else {
            throw Error(ERR_STATE, "detour DAG edge is not straight");
        }
        connect_pre(p, m1, slot);
        connect_pre(m1, m2, 0);
        connect_pre(m2, c, 0);
    }

    int displace(int q, int dir, int reg) {
        int a = 0;
        for (int s : stems[dir][reg]) a += std::abs(s - q);
        return a;
    }

    std::vector<int> mirror_places(int t, int dir) {
        const int v = P[t];
        const int reg = region[dir][t];
        const int cx = px_(v), cy = py_(v);
        const int trunk = range[dir][reg].second - range[dir][reg].first;
        const int maxd = (int)(ratio * (float)trunk);
        const int orig = dir ? cx : cy;
        const int od = displace(orig, dir, reg);
        int lo = orig, hi = orig;
        const int bound = dir ? X : Y;
        while (lo - 1 >= 0 && displace(lo - 1, dir, reg) - od <= maxd) lo--;
        while (hi + 1 < bound && displace(hi - 1, dir, reg) - od <= maxd) hi++;
        int step = 1;
        while ((orig - lo) / (step + 1) + (hi - orig) / (step + 1) >= num_tracks) step++;
        lo = orig - (orig - lo) / step * step;
        hi = orig + (hi - orig) / step * step;
        std::vector<int> sh;
        for (double pos = lo; pos <= hi; pos += step) {
            int s = (int)(pos - orig);
            if (s == 0) continue;
            sh.push_back((int)pos);
        }
        return sh;
    }

    void dfs(int x, int par, int par_node, int slot, int depth, const std::vector<std::vector<int>> &mirrors_in,
             const std::vector<std::vector<int>> &old_places) {
        static const std::vector<std::vector<int>> kNone(2);
        const std::vector<std::vector<int>> &mirrors = mirrors_in.empty() ? kNone : mirrors_in;
        const int v = P[x];
        const int cl = v / XY, cx = px_(v), cy = py_(v);
        const int me = create(cl, cx, cy);
        std::vector<std::vector<int>> new_mirrors(2), places(2);
        if (old_places.size() == 2) {
            for (int dir = 0; dir < 2; dir++) {
                const int rid = region_of(region[dir][x], dir);
                if (rid < 0) continue;
                if (region_of(region[dir][par], dir) == par) depth += 2;
                places[dir] = (x == rid) ? mirror_places(x, dir) : old_places[dir];
                if (rid != x && places[dir].size() != mirrors[dir].size())
                    throw Error(ERR_STATE, "mirror count mismatch in detour DAG");
                for (size_t m = 0; m < places[dir].size(); m++) {
                    const int nx = dir ? places[dir][m] : cx, ny = dir ? cy : places[dir][m];
                    int nm;
                    if (rid != x) {
                        nm = create(9, nx, ny);
                        connect(mirrors[dir][m], nm, slot);
                    } else if (x != root) {
                        const int pxx = px_(nodes[par_node]), pyy = py_(nodes[par_node]);
                        if (nx != pxx && ny != pyy) {
                            int tmp[2];
                            for (int pi = 0; pi <= 1; pi++) {
                                const int mx = pi ? nx : pxx, my = pi ? pyy : ny;
                                tmp[pi] = create(9, mx, my);
                                connect(par_node, tmp[pi], slot);
                            }
                            nm = create(9, nx, ny);
                            for (int t : tmp) connect(t, nm, 0);
                        } else {
                            nm = create(9, nx, ny);
                            connect(par_node, nm, slot);
                        }
                    } else {
                        nm = create(9, nx, ny);
                    }
                    new_mirrors[dir].push_back(nm);
                }
            }
        }
        if (par_node != -1) {
            const int ppx = px_(nodes[par_node]), ppy = py_(nodes[par_node]);
            if (ppx != cx && ppy != cy) {
                for (int pi = 0; pi <= 1; pi++) {
                    const int mx = pi ? cx : ppx, my = pi ? ppy : cy;
                    const int pre = create(9, mx, my);
                    connect(par_node, pre, slot);
                    connect(pre, me, 0);
                }
                for (int pi = 0; pi <= 1; pi++) {
                    const int len = pi ? std::abs(ppy - cy) : std::abs(ppx - cx);
                    int zs = 10, sel = 10;
                    if (mode == 0 || mode == 1) { zs = 7; sel = 2; }
                    const int mz = std::min(zs, len);
                    std::pair<float, int> road[10];  // value-initialised: (0, 0)
                    auto mids = [&](int k, int &x1, int &y1, int &x2, int &y2) {
                        x1 = pi ? ppx : (ppx * k + cx * (mz - k)) / mz;
                        y1 = pi ? (ppy * k + cy * (mz - k)) / mz : ppy;
                        x2 = pi ? cx : (ppx * k + cx * (mz - k)) / mz;
                        y2 = pi ? (ppy * k + cy * (mz - k)) / mz : cy;
                        if (x1 < 0 || y1 < 0 || x1 >= X || y1 >= Y) return false;
                        if (x1 == ppx && y1 == ppy) return false;
                        if (x1 == cx && y1 == cy) return false;
                        if (x2 < 0 || y2 < 0 || x2 >= X || y2 >= Y) return false;
                        if (x2 == cx && y2 == cy) return false;
                        if (x2 == ppx && y2 == ppy) return false;
                        return true;
                    };
                    for (int k = 1; k < mz; k++) {
                        int x1, y1, x2, y2;
                        if (!mids(k, x1, y1, x2, y2)) continue;
                        int of = 0;
                        of += ys(std::max(x1, x2), std::max(y1, y2)) - ys(std::min(x1, x2), std::min(y1, y2));
                        of += ys(std::max(x1, ppx), std::max(y1, ppy)) - ys(std::min(x1, ppx), std::min(y1, ppy));
                        of += ys(std::max(cx, x2), std::max(cy, y2)) - ys(std::min(cx, x2), std::min(cy, y2));
                        road[k - 1] = std::make_pair((float)of, k);
                    }
                    // ascending (the entries are distinct or equal as pairs, so any sort agrees)
                    for (int a = 1; a < mz - 1; a++)
                        for (int b = a; b > 0 && road[b] < road[b - 1]; b--) std::swap(road[b], road[b - 1]);
                    for (int ii = 0; ii < sel; ii++) {
                        const int k = road[ii].second;
                        int x1, y1, x2, y2;
                        if (mz == 0 || !mids(k, x1, y1, x2, y2)) continue;
                        const int p1 = create(9, x1, y1);
                        connect(par_node, p1, slot);
                        points.push_back((x1 + x2) / 2 * Y + (y1 + y2) / 2);
                        const int p2 = create(9, x2, y2);
                        connect(p1, p2, 0);
                        connect(p2, me, 0);
                    }
                }
            }
            for (int dir = 0; dir < 2; dir++) {
                const int rid = region_of(region[dir][x], dir);
                const int prid = region_of(region[dir][par], dir);
                if (prid >= 0 && rid != prid) {
                    for (int pm : mirrors[dir]) {
                        const int mx0 = px_(nodes[pm]), my0 = py_(nodes[pm]);
                        if (mx0 != cx && my0 != cy) {
                            for (int pi = 0; pi <= 1; pi++) {
                                const int mx = pi ? cx : mx0, my = pi ? my0 : cy;
                                const int ni = create(9, mx, my);
                                connect(pm, ni, slot);
                                connect(ni, me, 0);
                            }
                        } else {
                            connect(pm, me, slot);
                        }
                    }
                }
            }
            if (ppx == cx || ppy == cy) connect(par_node, me, slot);
        }
        for (int dir = 0; dir < 2; dir++) {
            const int rid = region_of(x, dir);
            if (rid < 0) continue;
            const bool is_pin = cl < 9;
            if (x != root && is_pin)
                for (int mid : new_mirrors[dir]) {
                    const int dup = create(cl, cx, cy);
                    connect(mid, dup, (int)G[x].size() - 1);
                }
        }
        int idx = 0;
        for (int e : G[x]) {
            if (e == par) continue;
            dfs(e, x, me, idx++, depth + 1, new_mirrors, places);
        }
    }

    void build() {
        root = select_root();
        if (root < 0) throw Error(ERR_STATE, "net tree without leaves");
        for (int dir = 0; dir < 2; dir++) {
            region[dir].assign(ntree, -1);
            range[dir].assign(ntree, {0, 0});
            if ((int)stems[dir].size() < ntree) stems[dir].resize(ntree);
            for (int i = 0; i < ntree; i++) stems[dir][i].clear();
        }
        for (int x = 0; x < ntree; x++) {
            const int v = P[x], cl = v / XY, cx = px_(v), cy = py_(v);
            for (int dir = 0; dir < 2; dir++) {
                if (cl < 9) stems[dir][x].push_back(dir ? cx : cy);
                const int t = dir ? cy : cx;
                range[dir][x] = {t, t};
            }
        }
        mark(root, -1);
        dfs(root, -1, -1, -1, 0, {}, {});
        std::sort(points.begin(), points.end());
        points.erase(std::unique(points.begin(), points.end()), points.end());
        // renumber: a node is placed once all of its children are placed (post order
        // on a stack), then popped so that parents precede children (:2027-2085)
        const int cnt = (int)nodes.size();
        // parents of every node in creation order (CSR)
        std::vector<int> &poff = sc.poff, &pcode = sc.pcode, &at = sc.at;
        poff.assign(cnt + 1, 0);
        pcode.resize(links.size());
        for (auto &l : links) poff[l.first + 1]++;
        for (int i = 0; i < cnt; i++) poff[i + 1] += poff[i];
        at.assign(poff.begin(), poff.end() - 1);
        for (auto &l : links) pcode[at[l.first]++] = l.second;
        std::vector<int> &visit = sc.visit, &newid = sc.newid, &stk = sc.stk;
        visit.assign(cnt, 0);
        newid.assign(cnt, 0);
        stk.clear();
        std::vector<std::pair<int, int>> &st = sc.st;
        for (int i = 0; i < cnt; i++) {
            if (child_pre[i] != 0) continue;
            // iterative form of determinSequence: push i, then every parent whose
            // children are all pushed, depth first in parent order
            st.clear();
            stk.push_back(i);
            st.push_back({i, poff[i]});
            while (!st.empty()) {
                auto &f = st.back();
                if (f.second >= poff[f.first + 1]) { st.pop_back(); continue; }
                const int p = pcode[f.second++] / 10;
                if (++visit[p] == child_pre[p]) {
                    stk.push_back(p);
                    st.push_back({p, poff[p]});
                }
            }
        }
        if ((int)stk.size() != cnt) throw Error(ERR_STATE, "detour DAG is not acyclic");
        out.nodes.assign(cnt, 0);
        out.par_num.assign(cnt, 0);
        out.par_sum.assign(cnt + 1, 0);
        out.child_num.assign(cnt, 0);
        out.depth.assign(cnt, 0);
        out.par_nodes.clear();
        out.child_idx.clear();
        int k = 0;
        while (!stk.empty()) {
            const int idx = stk.back();
            stk.pop_back();
            for (int q = poff[idx]; q < poff[idx + 1]; q++) {
                const int c = pcode[q];
                const int p = c / 10, sl = c % 10;
                const int sp = newid[p];
                out.child_num[sp] = std::max(out.child_num[sp], sl + 1);
                out.par_nodes.push_back(sp);
                out.child_idx.push_back(sl);
                out.depth[k] = std::max(out.depth[k], out.depth[sp] + 1);
            }
            newid[idx] = k;
            out.par_num[k] = poff[idx + 1] - poff[idx];
            out.par_sum[k + 1] = out.par_sum[k] + out.par_num[k];
            out.nodes[k] = nodes[idx];
            k++;
        }
        out.points.assign(points.begin(), points.end());
    }
};

}  // namespace

void build_dag(const NetSet &ns, const RNet &n, const CongestionView &cv, int mode, DagNet &out) {
    thread_local Scratch scratch;
    // the arrays are rewritten below; out keeps its memory resource
    out.par_nodes.clear();
    out.child_idx.clear();
    out.points.clear();
    Builder b(ns, n, cv, mode, out, scratch);
    b.build();
}

}  // namespace igr
