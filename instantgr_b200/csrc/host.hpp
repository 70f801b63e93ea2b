// Host-side data model of the global router: the parsed ISPD2024 design,
// the routing nets derived from it, and the helpers shared by the host
// passes (parser, pin selection, Steiner provider, net splitting, detour DAG
// construction, route-guide writer).
//
// Encodings kept identical to InstantGR so that routes, pins and trees can be
// exchanged with it verbatim:
//   * a 3-D position is  l*X*Y + x*Y + y   (src/database.hpp:36)
//   * a 2-D position is  x*Y + y
//   * "file" layers are 0..L-1 (L=10, layer 0 pin-only); "routing" layers are
//     file layer - 1 (src/database_cuda.hpp:2106, 2267), so routing layer r has
//     direction (r & 1) ^ DIR with DIR = direction of file layer 1.
#pragma once
#include <cstdint>
#include <functional>
#include <memory>
#include <memory_resource>
#include <stdexcept>
#include <string>
#include <vector>

#include "status.hpp"

namespace igr {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------- design
struct Design {
    int L = 0, X = 0, Y = 0;               // file layers, grid size
    double unit_wire = 0, unit_via = 0;
    std::vector<double> short_cost;         // [L] overflow weight per layer
    std::vector<int> x_edge_len, y_edge_len; // [X-1], [Y-1]
    std::vector<int> dr_x, dr_y;            // cumulative coordinates [X], [Y]
    std::vector<int> dr2gr_x, dr2gr_y;      // inverse of dr_x / dr_y (-1 = no grid line)
    std::vector<int> layer_dir;             // [L] 0 = horizontal, 1 = vertical
    std::vector<double> layer_min_len;      // [L]
    std::vector<float> cap;                 // [L][X][Y] capacity (file layers)
    std::vector<double> cap_d;              // the capacities as read, kept only when one is not a float

    // nets as read: CSR net -> pins -> access points
    std::vector<char> name_pool;
    std::vector<int64_t> name_off;          // [N+1]
    std::vector<int64_t> pin_off;           // [N+1] into ap_off
    std::vector<int64_t> ap_off;            // [P+1] into ap
    std::vector<int> ap;                    // 3-D positions
    std::vector<int> bminx, bmaxx, bminy, bmaxy; // bbox of all access points

    // after pin selection (src/database.hpp:38-243)
    std::vector<int64_t> sel_off;           // [N+1]
    std::vector<int> sel;                   // chosen 3-D pin positions
    std::vector<int64_t> extra_off;         // [N+1]
    std::vector<int> extra;                 // pairs of 3-D positions (stacked pins)

    int num_nets() const { return (int)name_off.size() - 1; }
    std::string name(int n) const {
        return std::string(name_pool.data() + name_off[n], name_pool.data() + name_off[n + 1]);
    }
    int dir_routing(int r) const { return layer_dir[r + 1]; }
};

// Reads the .cap and .net files with the semantics of InstantGR's scanner
// (src/database.hpp:247-409): digits only (no signs, no exponents), '.' as the
// only fraction mark, access points "(l, x, y)" grouped in "[...]" pins.
void read_design(Design &d, const char *cap_path, const char *net_path, int threads);
void read_cap_buffer(Design &d, const char *buf, size_t n, int threads = 0);
void read_net_buffer(Design &d, const char *buf, size_t n);

// Chooses one access point per pin (src/database.hpp:38-243), fills sel/extra.
void select_pins(Design &d, int threads);

// ---------------------------------------------------------------- routing nets
// Adjacency of a tree in CSR form: the neighbours of node i are
// nb[off[i] .. off[i+1]), in the order the edges were added.
struct TreeAdj {
    std::pmr::vector<int> off, nb;
    explicit TreeAdj(std::pmr::memory_resource *r = std::pmr::get_default_resource()) : off(1, 0, r), nb(r) {}
    struct Row {
        const int *b, *e;
        const int *begin() const { return b; }
        const int *end() const { return e; }
        size_t size() const { return (size_t)(e - b); }
        int operator[](size_t k) const { return b[k]; }
    };
    int size() const { return (int)off.size() - 1; }
    Row operator[](int i) const { return Row{nb.data() + off[i], nb.data() + off[i + 1]}; }
    // n nodes; each undirected edge (a, b) in order appends b to a's list, then a to b's
    void from_edges(int n, const std::vector<std::pair<int, int>> &edges);
};

// A routing net ("subnet") is a net of >= 2 selected pins, split at
// MAX_PIN_SIZE = 12 pins along its Steiner tree (src/database_cuda.hpp:2111-2237).
// Its arrays come from the memory resource it is made with (the net set's pool,
// so that a whole net set is freed at once).
struct RNet {
    int orig = -1;                 // design net id
    int hpwl = 0, minx = 0, maxx = 0, miny = 0, maxy = 0;
    std::pmr::vector<int> pins;    // routing-layer 3-D positions
    // Steiner tree: adjacency over nodes, node positions (3-D, Steiner -> layer L)
    TreeAdj adj;
    std::pmr::vector<int> tnode;
    explicit RNet(std::pmr::memory_resource *r = std::pmr::get_default_resource()) : pins(r), adj(r), tnode(r) {}
};

// 2-D conflict shapes of a routing net for batch colouring (net::construct_rsmt,
// src/database_cuda.hpp:746-820), in the reference's order: the tree nodes as
// points, then per tree edge (i, j < i) its horizontal and vertical segments
// (pairs of 2-D cells, lower first) and its end or corner points.
template <class Pt, class Hs, class Vs>
void for_each_shape(const RNet &n, int X, int Y, Pt &&point, Hs &&hseg, Vs &&vseg) {
    const int XY = X * Y;
    const int m = (int)n.tnode.size();
    for (int i = 0; i < m; i++) point(n.tnode[i] % XY);
    for (int i = 0; i < m; i++) {
        const int pi = n.tnode[i] % XY, xi = pi / Y, yi = pi % Y;
        for (int j : n.adj[i]) {
            if (j >= i) continue;
            const int pj = n.tnode[j] % XY, xj = pj / Y, yj = pj % Y;
            const int mnx = xi < xj ? xi : xj, mxx = xi < xj ? xj : xi;
            const int mny = yi < yj ? yi : yj, mxy = yi < yj ? yj : yi;
            if (xi != xj && yi != yj) {
                hseg(mnx * Y + mny, mxx * Y + mny);
                hseg(mnx * Y + mxy, mxx * Y + mxy);
                vseg(mnx * Y + mny, mnx * Y + mxy);
                vseg(mxx * Y + mny, mxx * Y + mxy);
                point(xi * Y + yj);
                point(xj * Y + yi);
            } else if (xi != xj) {
                hseg(mnx * Y + mny, mxx * Y + mny);
                point(mnx * Y + mny);
                point(mxx * Y + mny);
            } else if (yi != yj) {
                vseg(mnx * Y + mny, mnx * Y + mxy);
                point(mnx * Y + mny);
                point(mnx * Y + mxy);
            }
        }
    }
}

struct NetSet {
    int L = 0, X = 0, Y = 0, DIR = 0;   // routing layers (L = 9)
    // the nets' arrays: one arena per range of design nets, filled by one thread
    // at a time and freed as a whole (declared before the nets: freed after them)
    std::vector<std::unique_ptr<std::pmr::monotonic_buffer_resource>> arenas;
    std::vector<RNet> nets;
    std::vector<int> sub_off;                // [design nets + 1]: routing nets sub_off[n] .. sub_off[n+1]
    std::vector<int> unfinished;             // design net -> subnets still routing
    std::vector<int64_t> pin_sum;            // [n+1] pin prefix sum (route slots)
};

// Builds routing nets: Steiner trees for every multi-pin net, split >12-pin nets.
void build_netset(const Design &d, NetSet &ns, int threads);
// Tree (adj, tnode with layers) of one net (construct_rsmt, src/database_cuda.hpp:746-820).
void construct_rsmt(const Design &d, const NetSet &ns, RNet &n);
void calc_hpwl(const NetSet &ns, RNet &n);

// DFS preorder flattening of a tree (src/Lshape_route.hpp:191-208).
void flatten_tree(const RNet &n, int *nodes, int *par);

// ---------------------------------------------------------------- detour DAG
// Per-net detour DAG (src/database_cuda.hpp:1429-2086), in topological order.
// Its arrays come from the memory resource it is made with.
struct DagNet {
    std::pmr::vector<int> nodes;      // 3-D positions (routing layer; virtual = 9)
    std::pmr::vector<int> par_num;    // parents per node
    std::pmr::vector<int> par_sum;    // [n+1]
    std::pmr::vector<int> par_nodes;  // parent node (local index) per parent slot
    std::pmr::vector<int> child_idx;  // child slot of this node in the parent
    std::pmr::vector<int> child_num;  // children per node
    std::pmr::vector<int> depth;      // depth per node
    std::pmr::vector<int> points;     // 2-D conflict points
    explicit DagNet(std::pmr::memory_resource *r = std::pmr::get_default_resource())
        : nodes(r), par_num(r), par_sum(r), par_nodes(r), child_idx(r), child_num(r), depth(r), points(r) {}
};
struct CongestionView {            // host copy of the 2-D congestion prefix sums
    int X = 0, Y = 0;
    std::vector<float> xsum, ysum;
};
void build_dag(const NetSet &ns, const RNet &n, const CongestionView &cv, int mode, DagNet &out);
// Process-wide cache of host memory blocks for arenas: blocks given back stay
// mapped and are handed out again (powers of two), so that arenas made one
// after another reuse their pages.
std::pmr::memory_resource *host_block_cache();

// ---------------------------------------------------------------- Steiner provider
// Rectilinear Steiner tree of a point set; deterministic and independent of the
// input order.  Returns node positions (first the distinct input points in
// ascending (x, y) order, then Steiner points) and tree edges.
struct SteinerTree {
    std::vector<int> x, y;
    std::vector<std::pair<int, int>> edges;
};
void steiner_tree(const std::vector<int> &x, const std::vector<int> &y, SteinerTree &t);

// ---------------------------------------------------------------- output
// Writes route guides in InstantGR's order and format (src/graph.hpp:179-235).
struct RouteSource {
    // For routing net i: pointer to its route record (count at [0], then pairs).
    std::function<const int *(int)> routes_of;
};
void write_guides(const Design &d, const NetSet &ns, const RouteSource &rs, const char *path, int threads);

// ---------------------------------------------------------------- generator
struct GenParams {
    int X = 256, Y = 256, nets = 20000;
    uint64_t seed = 1;
    int cap_mode = 0;          // 0: U{4..12}; 1: mean falls 10 -> 4 over layers, +-2
    double block_frac = 0.05;  // fraction of routing edges zeroed in blockages
    int pin_mode = 0;          // 0: geometric(p=.5, min 2, cap 64); 1: mixture 70/20/9.5/0.5
    double hifanout_frac = 0;  // fraction of nets with 65..500 pins (pin_mode 0)
    int hifanout_bbox = 200;
    double bbox_median = 8, bbox_sigma = 1.0;
    int hotspots = 0;          // Gaussian hotspots
    double hotspot_frac = 0;   // fraction of nets centred on a hotspot
    double hotspot_sigma = 0;  // GCells
    // window written (0 x 0: the whole grid): the design is drawn in full, and
    // only the capacities of the window and the nets whose access points all
    // lie in it are written, shifted to the window's origin
    int win_x0 = 0, win_y0 = 0, win_w = 0, win_h = 0;
};
void generate_design(const GenParams &p, const char *cap_path, const char *net_path);
// parameters of the benchmark configurations 0..4 (nets scaled by `scale`)
GenParams config_params(int cfg, uint64_t seed, double scale);
GenParams custom_params(int X, int Y, int nets, uint64_t seed, int cap_mode, double block_frac, int pin_mode,
                        double hifanout_frac, double bbox_median, double bbox_sigma, int hotspots, double hotspot_frac);

int hw_threads();
void parallel_for(int n, int threads, const std::function<void(int, int)> &fn);  // fn(begin, end)
double now_s();

}  // namespace igr
