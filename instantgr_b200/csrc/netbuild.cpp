// Routing-net construction: Steiner trees, splitting of nets with more than
// 12 pins, conflict shapes for batch colouring, and tree flattening.
//
// Restates, in this project's own code, the host steps of InstantGR:
//   build_cuda_database's net split       src/database_cuda.hpp:2111-2237
//   my_flute (tree -> GCell graph, MST)   src/database_cuda.hpp:696-744
//   net::construct_rsmt (tree, layers)    src/database_cuda.hpp:746-820
//   net::calc_hpwl                        src/database_cuda.hpp:93-103
//   the DFS flattening of phase 1         src/Lshape_route.hpp:191-208
// The unstable std::sort calls of the reference (edges keyed on a single
// field) are reproduced with the same comparator on the same sequence, so the
// split is the same as the reference's for the same tree.
#include "host.hpp"
#include "steiner_core.hpp"

#include <algorithm>
#include <mutex>
#include <new>
#include <numeric>
#include <tuple>
#include <unordered_map>
#include <unordered_set>

namespace igr {

namespace {

// Tree over the distinct 2-D positions of `pos2d` (my_flute, database_cuda.hpp:696-744).
void tree_from_positions(const Design &d, int Y, const std::vector<int> &pos2d, TreeAdj &graph,
                         std::pmr::vector<int> &nodes) {
    // containers of one tree, kept per thread
    struct Scratch {
        std::vector<int> x, y, parent;
        igr_steiner::Tree t;
        std::vector<igr_steiner::Branch> br;
        std::vector<std::tuple<int, int, int>> edges;
        std::vector<uint64_t> ekey, etmp;
        std::vector<std::pair<int, int>> kept;
    };
    thread_local Scratch sc;
    std::vector<int> &x = sc.x, &y = sc.y;
    x.clear(); y.clear();
    for (int e : pos2d) { x.push_back(d.dr_x[e / Y]); y.push_back(d.dr_y[e % Y]); }
    const int cnt = (int)pos2d.size();
    igr_steiner::Tree &t = sc.t;
    igr_steiner::build(x, y, t);
    std::vector<igr_steiner::Branch> &br = sc.br;
    igr_steiner::to_branches(x, y, t, br);
    const int nb = 2 * cnt - 2;
    nodes.clear();
    for (int i = 0; i < nb; i++) nodes.push_back(d.dr2gr_x[br[i].x] * Y + d.dr2gr_y[br[i].y]);
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    std::vector<std::tuple<int, int, int>> &edges = sc.edges;
    edges.clear();
    auto where = [&](int g) { return (int)(std::lower_bound(nodes.begin(), nodes.end(), g) - nodes.begin()); };
    for (int i = 0; i < nb; i++)
        if (br[i].n < nb) {
            const auto &b1 = br[i], &b2 = br[b1.n];
            int u = where(d.dr2gr_x[b1.x] * Y + d.dr2gr_y[b1.y]);
            int v = where(d.dr2gr_x[b2.x] * Y + d.dr2gr_y[b2.y]);
            if (u == v) continue;
            edges.emplace_back(std::abs(b1.x - b2.x) + std::abs(b1.y - b2.y), u, v);
        }
    if (edges.size() >= 256 && nodes.size() <= 65536) {
        // (length, u, v) as one key that sorts as the triple does (lengths
        // and node indices are non-negative, indices below 2^16)
        std::vector<uint64_t> &ek = sc.ekey;
        ek.resize(edges.size());
        for (size_t i = 0; i < edges.size(); i++)
            ek[i] = (uint64_t)(uint32_t)std::get<0>(edges[i]) << 32 | (uint64_t)std::get<1>(edges[i]) << 16 |
                    (uint64_t)std::get<2>(edges[i]);
        igr_steiner::sort_keys(ek, sc.etmp);
        for (size_t i = 0; i < edges.size(); i++)
            edges[i] = {(int)(ek[i] >> 32), (int)(ek[i] >> 16 & 0xffff), (int)(ek[i] & 0xffff)};
    } else {
        std::sort(edges.begin(), edges.end());
    }
    std::vector<int> &parent = sc.parent;
    parent.resize(nodes.size());
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int v) {
        int r = v;
        while (parent[r] != r) r = parent[r];
        while (parent[v] != r) { const int n = parent[v]; parent[v] = r; v = n; }
        return r;
    };
    std::vector<std::pair<int, int>> &kept = sc.kept;
    kept.clear();
    for (auto &e : edges) {
        int u = std::get<1>(e), v = std::get<2>(e), pu = find(u), pv = find(v);
        if (pu != pv) {
            kept.push_back({u, v});
            parent[pu] = pv;
        }
    }
    graph.from_edges((int)nodes.size(), kept);
}

// Upstream of the net arenas: blocks given back stay mapped and are handed out
// again (rounded up to powers of two), so that the next design opened in this
// process reuses them instead of faulting in new pages.
class BlockCache final : public std::pmr::memory_resource {
    std::mutex mu_;
    std::vector<std::vector<void *>> free_;  // by log2 of the block size
    static int cls(size_t b) {
        int c = 12;
        while (((size_t)1 << c) < b) c++;
        return c;
    }
    void *do_allocate(size_t bytes, size_t align) override {
        const int c = cls(std::max(bytes, align));
        {
            std::lock_guard<std::mutex> lock(mu_);
            if (c < (int)free_.size() && !free_[c].empty()) {
                void *p = free_[c].back();
                free_[c].pop_back();
                return p;
            }
        }
        return ::operator new((size_t)1 << c, std::align_val_t(std::max<size_t>(align, 64)));
    }
    void do_deallocate(void *p, size_t bytes, size_t align) override {
        const int c = cls(std::max(bytes, align));
        std::lock_guard<std::mutex> lock(mu_);
        if ((int)free_.size() <= c) free_.resize(c + 1);
        free_[c].push_back(p);
    }
    bool do_is_equal(const std::pmr::memory_resource &o) const noexcept override { return this == &o; }
};

}  // namespace

std::pmr::memory_resource *host_block_cache() {
    static BlockCache *c = new BlockCache;  // never destroyed: arenas may outlive static destruction
    return c;
}

void TreeAdj::from_edges(int n, const std::vector<std::pair<int, int>> &edges) {
    off.assign(n + 1, 0);
    for (auto &e : edges) { off[e.first + 1]++; off[e.second + 1]++; }
    for (int i = 0; i < n; i++) off[i + 1] += off[i];
    nb.resize(off[n]);
    std::vector<int> at(off.begin(), off.end() - 1);
    for (auto &e : edges) {
        nb[at[e.first]++] = e.second;
        nb[at[e.second]++] = e.first;
    }
}

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

void construct_rsmt(const Design &d, const NetSet &ns, RNet &n) {
    const int X = ns.X, Y = ns.Y, XY = X * Y, L = ns.L;
    if (n.pins.size() == 2 && n.tnode.empty()) {
        // two pins: the provider's tree is the one edge between them whatever
        // the input order (FLUTE's degree-2 branches), so the nodes are the two
        // GCells in ascending order, each the other's neighbour
        const int a = n.pins[0], b = n.pins[1];
        if (a % XY == b % XY) throw Error(ERR_STATE, "two pins of a routing net share a 2-D position");
        const int lo = a % XY < b % XY ? a : b, hi = lo == a ? b : a;
        n.tnode.assign({lo, hi});
        n.adj.off.assign({0, 1, 2});
        n.adj.nb.assign({1, 0});
        return;
    }
    // pins are distinct in 2-D (checked below); the layer of each 2-D position
    thread_local std::vector<std::pair<int, int>> layer;
    thread_local std::vector<int> pos;
    layer.clear();
    pos.clear();
    // my_flute hands FLUTE the 2-D positions in the iteration order of a
    // std::unordered_set (src/database_cuda.hpp:696-708, 746-756).  The tree
    // does not depend on that order here: the provider sorts its points, and
    // tree_from_positions keys every edge by its GCells and sorts the edges
    // completely, so the positions go in pin order.
    for (int p : n.pins) {
        layer.push_back({p % XY, p / XY});
        pos.push_back(p % XY);
    }
    std::sort(layer.begin(), layer.end());
    for (size_t i = 1; i < layer.size(); i++)
        if (layer[i].first == layer[i - 1].first)
            throw Error(ERR_STATE, "two pins of a routing net share a 2-D position");
    if (n.tnode.empty()) {
        tree_from_positions(d, Y, pos, n.adj, n.tnode);
    } else {
        for (auto &e : n.tnode) e %= XY;
    }
    for (auto &e : n.tnode) {
        auto it = std::lower_bound(layer.begin(), layer.end(), std::make_pair(e, -1));
        e += (it != layer.end() && it->first == e ? it->second : L) * XY;
    }
}

namespace {

// Splits one design net with more than MAX_PIN_SIZE pins along its tree
// (database_cuda.hpp:2130-2228).
void split_net(const Design &d, const NetSet &ns, int db_id, std::vector<RNet> &out) {
    std::pmr::memory_resource *res = std::pmr::get_default_resource();
    const int MAX_PIN_SIZE = 12;
    const int X = ns.X, Y = ns.Y, XY = X * Y, L = ns.L;
    // containers of one split, kept per thread
    struct Scratch {
        RNet tmp;
        std::vector<char> not_steiner;
        std::vector<int> sz, par;
        std::vector<std::tuple<int, int, int>> edges;
        std::vector<std::vector<int>> new_pins, net_edge;
        std::vector<std::pair<int, int>> se;
    };
    thread_local Scratch sc;
    RNet &tmp = sc.tmp;
    tmp.pins.clear();
    tmp.tnode.clear();
    for (int64_t i = d.sel_off[db_id]; i < d.sel_off[db_id + 1]; i++) {
        int p = d.sel[i];
        tmp.pins.push_back(p >= XY ? p - XY : p);
    }
    tmp.orig = db_id;
    construct_rsmt(d, ns, tmp);
    const auto &tn = tmp.tnode;
    const int n = (int)tn.size();
    std::vector<char> &not_steiner = sc.not_steiner;
    not_steiner.resize(n);
    for (int i = 0; i < n; i++) not_steiner[i] = tn[i] < L * XY;
    std::vector<int> &sz = sc.sz, &par = sc.par;
    sz.assign(n, 1);
    par.resize(n);
    std::vector<std::tuple<int, int, int>> &edges = sc.edges;
    edges.clear();
    auto find = [&](int v) {
        int r = v;
        while (par[r] != r) r = par[r];
        while (par[v] != r) { const int q = par[v]; par[v] = r; v = q; }
        return r;
    };
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
    std::vector<std::vector<int>> &new_pins = sc.new_pins, &net_edge = sc.net_edge;
    if ((int)new_pins.size() < n) {
        new_pins.resize(n);
        net_edge.resize(n);
    }
    for (int i = 0; i < n; i++) {
        new_pins[i].clear();
        net_edge[i].clear();
    }
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
        RNet s(res);
        s.orig = db_id;
        const std::vector<int> &np = new_pins[i];
        for (int j = 0; j < (int)np.size(); j++)
            if (np[j] < L * XY) s.pins.push_back(np[j]);
        // index of a node in the subnet: its last position in np (a map filled
        // in order keeps the last)
        auto index_of = [&](int v) {
            for (int j = (int)np.size() - 1; j >= 0; j--)
                if (np[j] == v) return j;
            return 0;  // every edge end is in np
        };
        s.tnode.assign(np.begin(), np.end());
        std::vector<std::pair<int, int>> &se = sc.se;
        se.clear();
        for (int j : net_edge[i]) {
            auto &e = edges[j];
            int u = std::get<0>(e), v = std::get<1>(e);
            if (find(v) == i) std::swap(u, v);
            se.push_back({index_of(tn[u]), index_of(tn[v])});
        }
        s.adj.from_edges((int)np.size(), se);
        out.push_back(std::move(s));
    }
}

}  // namespace

void build_netset(const Design &d, NetSet &ns, int threads) {
    ns.L = d.L - 1; ns.X = d.X; ns.Y = d.Y; ns.DIR = d.layer_dir[1];
    ns.nets.clear();
    ns.arenas.clear();
    const int N = d.num_nets(), XY = d.X * d.Y;
    if (threads <= 0) threads = hw_threads();
    // tasks: ranges of design nets, each with its own arena
    const int T = std::max(1, std::min(N, 8 * threads));
    for (int t = 0; t < T; t++)
        ns.arenas.push_back(std::make_unique<std::pmr::monotonic_buffer_resource>(host_block_cache()));
    auto task_begin = [&](int t) { return (int)((int64_t)N * t / T); };
    // nets of more than 12 pins are split first (in parallel); every other
    // multi-pin net is one routing net
    std::vector<int> big;
    for (int id = 0; id < N; id++)
        if (d.sel_off[id + 1] - d.sel_off[id] > 12) big.push_back(id);
    std::vector<std::vector<RNet>> parts(big.size());
    parallel_for((int)big.size(), threads, [&](int b, int e) {
        for (int k = b; k < e; k++) split_net(d, ns, big[k], parts[k]);
    });
    ns.unfinished.assign(N, 0);
    ns.sub_off.assign(N + 1, 0);
    for (int id = 0, k = 0; id < N; id++) {
        const int64_t np = d.sel_off[id + 1] - d.sel_off[id];
        const int cnt = np == 1 ? 0 : (np <= 12 ? 1 : (int)parts[k++].size());
        ns.unfinished[id] = cnt;
        ns.sub_off[id + 1] = ns.sub_off[id] + cnt;
    }
    const int R = ns.sub_off[N];
    ns.nets.clear();
    ns.nets.reserve(R);
    for (int t = 0; t < T; t++)
        for (int r = ns.sub_off[task_begin(t)]; r < ns.sub_off[task_begin(t + 1)]; r++)
            ns.nets.emplace_back(ns.arenas[t].get());
    std::vector<int> part_of(N, -1);
    for (int k = 0; k < (int)big.size(); k++) part_of[big[k]] = k;
    // routing nets in design-net order; trees of every routing net (Lshape_route.hpp:159-163)
    parallel_for(T, threads, [&](int tb, int te) {
        for (int id = task_begin(tb); id < task_begin(te); id++) {
            const int r0 = ns.sub_off[id], r1 = ns.sub_off[id + 1];
            if (r0 == r1) continue;
            if (part_of[id] >= 0) {
                auto &pv = parts[part_of[id]];
                for (int r = r0; r < r1; r++) ns.nets[r] = std::move(pv[r - r0]);
                // the split's own copies are freed here, on the worker threads,
                // not one by one on the calling thread when `parts` goes
                std::vector<RNet>().swap(pv);
            } else {
                RNet &r = ns.nets[r0];
                r.orig = id;
                r.pins.reserve(d.sel_off[id + 1] - d.sel_off[id]);
                for (int64_t i = d.sel_off[id]; i < d.sel_off[id + 1]; i++) {
                    int p = d.sel[i];
                    r.pins.push_back(p >= XY ? p - XY : p);
                }
            }
            for (int r = r0; r < r1; r++) {
                calc_hpwl(ns, ns.nets[r]);
                construct_rsmt(d, ns, ns.nets[r]);
            }
        }
    });
    ns.pin_sum.assign(R + 1, 0);
    for (int i = 0; i < R; i++) ns.pin_sum[i + 1] = ns.pin_sum[i] + (int64_t)ns.nets[i].pins.size();
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
    // slots of nodes the DFS did not reach (none for a connected tree) are
    // zeroed, since the caller's arrays start uninitialised
    for (int k = cnt; k < (int)n.tnode.size(); k++) nodes[k] = par[k] = 0;
}

}  // namespace igr
