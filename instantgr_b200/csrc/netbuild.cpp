// Routing-net construction: Steiner trees, splitting of nets with more than
// 12 pins, conflict shapes for batch colouring, and tree flattening.
//
// Restates, in this project's own code, the host steps of InstantGR:
//   build_cuda_database's net split       src/database_cuda.hpp:2111-2237
//   my_flute (tree -> GCell graph, MST)   src/database_cuda.hpp:696-744
//   net::construct_rsmt (segments/points) src/database_cuda.hpp:746-820
//   net::calc_hpwl                        src/database_cuda.hpp:93-103
//   the DFS flattening of phase 1         src/Lshape_route.hpp:191-208
// The unstable std::sort calls of the reference (edges keyed on a single
// field) are reproduced with the same comparator on the same sequence, so the
// split is the same as the reference's for the same tree.
#include "host.hpp"
#include "steiner_core.hpp"

#include <algorithm>
#include <numeric>
#include <tuple>
#include <unordered_map>

namespace igr {

namespace {

// Tree over the distinct 2-D positions of `pos2d` (my_flute, database_cuda.hpp:696-744).
void tree_from_positions(const Design &d, int Y, const std::vector<int> &pos2d,
                         std::vector<std::vector<int>> &graph, std::vector<int> &nodes) {
    std::vector<int> x, y;
    x.reserve(pos2d.size()); y.reserve(pos2d.size());
    for (int e : pos2d) { x.push_back(d.dr_x[e / Y]); y.push_back(d.dr_y[e % Y]); }
    const int cnt = (int)pos2d.size();
    igr_steiner::Tree t;
    igr_steiner::build(x, y, t);
    std::vector<igr_steiner::Branch> br;
    igr_steiner::to_branches(x, y, t, br);
    const int nb = 2 * cnt - 2;
    nodes.clear();
    for (int i = 0; i < nb; i++) nodes.push_back(d.dr2gr_x[br[i].x] * Y + d.dr2gr_y[br[i].y]);
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    std::vector<std::tuple<int, int, int>> edges;
    edges.reserve(nb);
    auto where = [&](int g) { return (int)(std::lower_bound(nodes.begin(), nodes.end(), g) - nodes.begin()); };
    for (int i = 0; i < nb; i++)
        if (br[i].n < nb) {
            const auto &b1 = br[i], &b2 = br[b1.n];
            int u = where(d.dr2gr_x[b1.x] * Y + d.dr2gr_y[b1.y]);
            int v = where(d.dr2gr_x[b2.x] * Y + d.dr2gr_y[b2.y]);
            if (u == v) continue;
            edges.emplace_back(std::abs(b1.x - b2.x) + std::abs(b1.y - b2.y), u, v);
        }
    std::sort(edges.begin(), edges.end());
    std::vector<int> parent(nodes.size());
    std::iota(parent.begin(), parent.end(), 0);
    std::function<int(int)> find = [&](int v) { return v == parent[v] ? v : parent[v] = find(parent[v]); };
    graph.assign(nodes.size(), {});
    for (auto &e : edges) {
        int u = std::get<1>(e), v = std::get<2>(e), pu = find(u), pv = find(v);
        if (pu != pv) {
            graph[u].push_back(v);
            graph[v].push_back(u);
            parent[pu] = pv;
        }
    }
}

}  // namespace

void steiner_tree(const std::vector<int> &x, const std::vector<int> &y, SteinerTree &t) {
    igr_steiner::Tree s;
    igr_steiner::build(x, y, s);
    t.x = s.x;
    t.y = s.y;
    t.edges = s.edges;
}

void calc_hpwl(const NetSet &ns, RNet &n) {
    const int X = ns.X, Y = ns.Y;
    n.minx = X; n.maxx = 0; n.miny = Y; n.maxy = 0;
    for (int p : n.pins) {
        int x = p / Y % X, y = p % Y;
        n.minx = std::min(n.minx, x); n.maxx = std::max(n.maxx, x);
        n.miny = std::min(n.miny, y); n.maxy = std::max(n.maxy, y);
    }
    n.hpwl = n.maxx - n.minx + n.maxy - n.miny;
}

void construct_rsmt(const Design &d, const NetSet &ns, RNet &n, bool rsmt_only) {
    const int X = ns.X, Y = ns.Y, XY = X * Y, L = ns.L;
    std::unordered_map<int, int> layer;
    std::vector<int> pos;
    for (int p : n.pins) {
        int q = p % XY;
        if (!layer.count(q)) pos.push_back(q);
        layer[q] = p / XY;
    }
    if (pos.size() != n.pins.size()) throw Error(ERR_STATE, "two pins of a routing net share a 2-D position");
    if (n.tnode.empty()) {
        tree_from_positions(d, Y, pos, n.adj, n.tnode);
    } else {
        for (auto &e : n.tnode) e %= XY;
    }
    if (!rsmt_only) {
        n.hseg.clear(); n.vseg.clear();
        n.points = n.tnode;
        for (int i = 0; i < (int)n.tnode.size(); i++) {
            int xi = n.tnode[i] / Y, yi = n.tnode[i] % Y;
            for (int j : n.adj[i]) {
                if (j >= i) continue;
                int xj = n.tnode[j] / Y, yj = n.tnode[j] % Y;
                int mnx = std::min(xi, xj), mxx = std::max(xi, xj), mny = std::min(yi, yj), mxy = std::max(yi, yj);
                if (xi != xj && yi != yj) {
                    n.hseg.push_back({mnx * Y + mny, mxx * Y + mny});
                    n.hseg.push_back({mnx * Y + mxy, mxx * Y + mxy});
                    n.vseg.push_back({mnx * Y + mny, mnx * Y + mxy});
                    n.vseg.push_back({mxx * Y + mny, mxx * Y + mxy});
                    n.points.push_back(xi * Y + yj);
                    n.points.push_back(xj * Y + yi);
                } else if (xi != xj) {
                    n.hseg.push_back({mnx * Y + mny, mxx * Y + mny});
                    n.points.push_back(mnx * Y + mny);
                    n.points.push_back(mxx * Y + mny);
                } else if (yi != yj) {
                    n.vseg.push_back({mnx * Y + mny, mnx * Y + mxy});
                    n.points.push_back(mnx * Y + mny);
                    n.points.push_back(mnx * Y + mxy);
                }
            }
        }
    }
    for (auto &e : n.tnode) {
        auto it = layer.find(e);
        e += (it != layer.end() ? it->second : L) * XY;
    }
}

namespace {

// Splits one design net with more than MAX_PIN_SIZE pins along its tree
// (database_cuda.hpp:2130-2228).
void split_net(const Design &d, const NetSet &ns, int db_id, std::vector<RNet> &out) {
    const int MAX_PIN_SIZE = 12;
    const int X = ns.X, Y = ns.Y, XY = X * Y, L = ns.L;
    RNet tmp;
    for (int64_t i = d.sel_off[db_id]; i < d.sel_off[db_id + 1]; i++) {
        int p = d.sel[i];
        tmp.pins.push_back(p >= XY ? p - XY : p);
    }
    tmp.orig = db_id;
    construct_rsmt(d, ns, tmp, true);
    const auto &tn = tmp.tnode;
    const int n = (int)tn.size();
    std::vector<char> not_steiner(n);
    for (int i = 0; i < n; i++) not_steiner[i] = tn[i] < L * XY;
    std::vector<int> sz(n, 1), par(n);
    std::vector<std::tuple<int, int, int>> edges;
    edges.reserve(n);
    std::function<int(int)> find = [&](int v) { return v == par[v] ? v : par[v] = find(par[v]); };
    for (int i = 0; i < n; i++) {
        par[i] = i;
        for (int j : tmp.adj[i])
            if (j < i) edges.emplace_back(j, i, not_steiner[i] + not_steiner[j]);
    }
    std::sort(edges.begin(), edges.end(),
              [](std::tuple<int, int, int> l, std::tuple<int, int, int> r) { return std::get<2>(l) < std::get<2>(r); });
    bool big_steiner = false;
    for (auto &e : edges) {
        int u = find(std::get<0>(e)), v = find(std::get<1>(e));
        if (u == v) continue;
        if (sz[u] + sz[v] > MAX_PIN_SIZE) {
            if (!(not_steiner[std::get<0>(e)] || not_steiner[std::get<1>(e)])) big_steiner = true;
            if (!big_steiner) continue;
        }
        if (sz[u] > sz[v]) std::swap(u, v);
        par[u] = v;
        sz[v] += sz[u];
    }
    std::vector<std::vector<int>> new_pins(n), net_edge(n);
    for (int i = 0; i < n; i++) new_pins[find(i)].push_back(tn[i]);
    for (int i = 0; i < (int)edges.size(); i++) {
        auto &e = edges[i];
        int u = std::get<0>(e), v = std::get<1>(e);
        int pu = find(u), pv = find(v);
        if (pu == pv) { net_edge[pu].push_back(i); continue; }
        if (sz[u] > sz[v]) { std::swap(u, v); std::swap(pu, pv); }
        if (!not_steiner[v] && not_steiner[u]) { std::swap(u, v); std::swap(pu, pv); }
        sz[pu]++;
        if (sz[pv] == 1) par[pv] = pu;
        net_edge[pu].push_back(i);
        new_pins[pu].push_back(tn[v]);
    }
    for (int i = 0; i < n; i++) {
        if (find(i) != i) continue;
        RNet s;
        s.orig = db_id;
        std::unordered_map<int, int> indx;
        for (int j = 0; j < (int)new_pins[i].size(); j++) {
            if (new_pins[i][j] < L * XY) s.pins.push_back(new_pins[i][j]);
            indx[new_pins[i][j]] = j;
        }
        s.adj.assign(new_pins[i].size(), {});
        s.tnode = new_pins[i];
        for (int j : net_edge[i]) {
            auto &e = edges[j];
            int u = std::get<0>(e), v = std::get<1>(e);
            if (find(v) == i) std::swap(u, v);
            int a = indx[tn[u]], b = indx[tn[v]];
            s.adj[a].push_back(b);
            s.adj[b].push_back(a);
        }
        out.push_back(std::move(s));
    }
}

}  // namespace

void build_netset(const Design &d, NetSet &ns, int threads) {
    ns.L = d.L - 1; ns.X = d.X; ns.Y = d.Y; ns.DIR = d.layer_dir[1];
    const int N = d.num_nets(), XY = d.X * d.Y;
    std::vector<std::vector<RNet>> tmp(N);
    ns.unfinished.assign(N, 0);
    parallel_for(N, threads, [&](int b, int e) {
        for (int id = b; id < e; id++) {
            int64_t np = d.sel_off[id + 1] - d.sel_off[id];
            if (np == 1) continue;
            if (np <= 12) {
                RNet r;
                r.orig = id;
                for (int64_t i = d.sel_off[id]; i < d.sel_off[id + 1]; i++) {
                    int p = d.sel[i];
                    r.pins.push_back(p >= XY ? p - XY : p);
                }
                tmp[id].push_back(std::move(r));
                ns.unfinished[id] = 1;
                continue;
            }
            split_net(d, ns, id, tmp[id]);
            ns.unfinished[id] = (int)tmp[id].size();
        }
    });
    ns.nets.clear();
    ns.subnets.assign(N, {});
    for (int id = 0; id < N; id++)
        for (auto &r : tmp[id]) {
            ns.subnets[id].push_back((int)ns.nets.size());
            ns.nets.push_back(std::move(r));
        }
    const int R = (int)ns.nets.size();
    parallel_for(R, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) calc_hpwl(ns, ns.nets[i]);
    });
    ns.pin_sum.assign(R + 1, 0);
    for (int i = 0; i < R; i++) ns.pin_sum[i + 1] = ns.pin_sum[i] + (int64_t)ns.nets[i].pins.size();
    // trees, segments and points of every routing net (Lshape_route.hpp:159-163)
    parallel_for(R, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) construct_rsmt(d, ns, ns.nets[i], false);
    });
}

void flatten_tree(const RNet &n, int *nodes, int *par) {
    int cnt = 0;
    // iterative DFS preorder that visits children in adjacency order
    struct F { int x, p, pidx; size_t k; };
    std::vector<F> st;
    st.push_back({0, -1, -1, 0});
    int idx0 = cnt++;
    nodes[idx0] = n.tnode[0];
    par[idx0] = -1;
    std::vector<int> myidx{idx0};
    while (!st.empty()) {
        F &f = st.back();
        if (f.k >= n.adj[f.x].size()) { st.pop_back(); myidx.pop_back(); continue; }
        int e = n.adj[f.x][f.k++];
        if (e == f.p) continue;
        int id = cnt++;
        nodes[id] = n.tnode[e];
        par[id] = myidx.back();
        int px = f.x;
        st.push_back({e, px, id, 0});
        myidx.push_back(id);
    }
    (void)cnt;
}

}  // namespace igr
