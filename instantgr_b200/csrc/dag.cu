// Phase-2 DAG routing: per-edge mid-edge layer changes, the level-by-level
// DAG DP, the backtrace with route emission and demand, and a deterministic
// compaction of the emitted routes.
//
// Restates, with the reference's arithmetic and tie rules:
//   precompute_cost_edge                  src/Lshape_route_detour.hpp:123-195
//   Lshape_route_node_layer_change_cuda   src/Lshape_route_detour.hpp:281-406
//   get_routing_tree_layer_change_cuda    src/Lshape_route_detour.hpp:520-694
//   cost/id packing for atomicMin         src/Lshape_route_detour.hpp:83-112
// The reference launches two kernels per DAG level of the whole batch, with a
// host synchronisation after each (2 x depth launches per batch).  The nets of
// a batch share no DAG node, so here one CTA walks one net's levels, bottom-up
// then top-down, separated by CTA barriers: one launch per batch and no grid
// synchronisation.  A warp computes the DP of one node; a thread traces one
// node.  Emitted segments are staged per DAG node and compacted in node order,
// so route records do not depend on atomic ordering (the reference appends
// them with atomicAdd).
#include "kcommon.cuh"

#include <algorithm>

namespace igr {

namespace {

constexpr int kML = 10;                      // MAX_LAYER of the reference
constexpr unsigned long long kInitPacked = 7208259049189261824ULL;  // init_cost_with_road
constexpr int kDagWarps = 8;                 // warps of one net's CTA
constexpr int kDagThreads = 32 * kDagWarps;
constexpr int kSmallWarps = 2;               // warps of a small net's CTA
constexpr int kSmallNodes = 64;              // a small net's DAG has at most this many nodes
constexpr int kSmallStageNodes = 96;         // nets staged with the smaller shared memory when a batch is split
constexpr int kBigWarps = 16;                // warps of the CTAs of the larger nets of a split batch

__device__ __forceinline__ int32_t f2o(float f) {
    int32_t i = __float_as_int(f);
    return (i >= 0) ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int32_t i) { return __int_as_float((i >= 0) ? i : i ^ 0x7FFFFFFF); }
__device__ __forceinline__ unsigned long long pack(float cost, int id) {
    return ((unsigned long long)f2o(cost) << 32) | (unsigned int)id;
}
__device__ __forceinline__ double packed_cost(unsigned long long p) { return (double)o2f((int32_t)(p >> 32)); }
__device__ __forceinline__ int packed_id(unsigned long long p) { return (int)(p & 0xFFFFFFFFull); }

__device__ __forceinline__ double wire_cost(const GridDev &g, int l, int xa, int xb, int ya, int yb) {
    return g.presum[cell_at(g, l, xb, yb)] - g.presum[cell_at(g, l, xa, ya)];
}

__device__ __forceinline__ void add_wire(const GridDev &g, int l, int xa, int xb, int ya, int yb, int stamp) {
    atomicAdd(&g.pre[cell_at(g, l, xa, ya)], 1);
    if (xa == xb) {
        atomicAdd(&g.pre[cell_at(g, l, xa, yb)], -1);
        g.stamp[cell_at(g, l, xa, yb)] = stamp;
    }
    if (ya == yb) {
        atomicAdd(&g.pre[cell_at(g, l, xb, ya)], -1);
        g.stamp[cell_at(g, l, xb, ya)] = stamp;
    }
    int first = 0;
    for (int k = 0; k < l; k++) first += layer_dir(g, k) ? g.X : g.Y;
    g.dirty_commit[first + (layer_dir(g, l) ? xa : ya)] = 1;
}

constexpr int kEdgeWarps = 4;
constexpr int kMaxPos = 40;  // mid-edge positions of one edge: at most 38 (see below)

struct EdgeScratch {
    double vc[kMaxPos][9];  // via cost per position and layer
    double ps[kMaxPos][9];  // wire prefix sum per position and layer
    double pf[9], pt[9];    // wire prefix sums at the child and the parent end
};

// precompute_cost_edge, one warp per edge.  For every source layer f whose
// direction runs along the edge and every target layer t of the same parity,
// the cheapest position of the layer change among the positions s0 + k * dd
// strictly inside the edge (dd = dist / min(dist, 20), so at most 38 of them):
// via cost of the column from min(f, t) to max(f, t) plus the wire costs of
// both legs, first minimum in position order.  Source layers across the edge
// get INF.  Only edges longer than 4 GCells are computed: the DP reads these
// costs for such edges alone, and the backtrace only where the DP chose them.
// The positions' via costs and prefix sums are staged in shared memory; each
// lane then scans the positions for one (f, t) pair with the reference's
// additions in the reference's order.
__global__ void __launch_bounds__(32 * kEdgeWarps) dag_edge_cost_kernel(GridDev g, DagBatchDev b) {
    chain_begin();
    __shared__ EdgeScratch scr[kEdgeWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * kEdgeWarps + warp;
    if (e >= b.n_edges) return;
    EdgeScratch &s = scr[warp];
    const int Y = g.Y, X = g.X;
    const int to_node = b.par[e], from_node = b.edge_child[e];
    const int tox = b.nodes[to_node] / Y % X, toy = b.nodes[to_node] % Y;
    const int fx = b.nodes[from_node] / Y % X, fy = b.nodes[from_node] % Y;
    const int dist = abs(tox - fx) + abs(toy - fy);
    if (dist <= 4) return;
    double *ce = b.cost_edges + e * 81;
    int *bc = b.best_change + e * 81;
    if (lane < 9) {
        const int f = lane;
        if ((layer_dir(g, f) == 0 && fy != toy) || (layer_dir(g, f) == 1 && fx != tox))
            for (int t = 0; t < 9; t++) ce[f * 9 + t] = kInf;
    }
    const bool vert = fx == tox;
    if (!vert && fy != toy) return;  // no source layer runs along a bent edge
    const int dd = dist / min(dist, 20);
    const int s0 = vert ? min(fy, toy) : min(fx, tox);
    const int npos = (dist - 1) / dd;  // positions s0 + k * dd < s0 + dist, k >= 1
    for (int i = lane; i < npos * 9; i += 32) {
        const int p = i / 9, l = i % 9;
        const int sp = s0 + (p + 1) * dd;
        const int sx = vert ? fx : sp, sy = vert ? sp : fy;
        const int64_t cell = cell_at(g, l, sx, sy);
        s.vc[p][l] = g.vcost[cell];
        s.ps[p][l] = g.presum[cell];
    }
    if (lane < 9) s.pf[lane] = g.presum[cell_at(g, lane, fx, fy)];
    else if (lane < 18) s.pt[lane - 9] = g.presum[cell_at(g, lane - 9, tox, toy)];
    __syncwarp();
    // the source layers along the edge are one parity class (directions
    // alternate): f0, f0 + 2, ...; pair i = (f0 + 2 (i / nv), f0 + 2 (i % nv))
    const int f0 = layer_dir(g, 0) == (vert ? 1 : 0) ? 0 : 1;
    const int nv = f0 == 0 ? 5 : 4;
    if (lane >= nv * nv) return;
    const int f = f0 + 2 * (lane / nv), t = f0 + 2 * (lane % nv);
    const int lo = min(f, t), hi = max(f, t);
    const int fa = vert ? fy : fx, ta = vert ? toy : tox;  // the ends along the edge
    double best = kInf;
    int pos = -1;
    for (int p = 0; p < npos; p++) {
        const int sp = s0 + (p + 1) * dd;
        double via = 0;
        for (int ll = lo; ll < hi; ll++) via += s.vc[p][ll];
        double c = via;
        const double wf = fa < sp ? s.ps[p][f] - s.pf[f] : s.pf[f] - s.ps[p][f];
        const double wt = ta < sp ? s.ps[p][t] - s.pt[t] : s.pt[t] - s.ps[p][t];
        c += (wf + wt);
        if (c < best) { best = c; pos = sp; }
    }
    ce[f * 9 + t] = best;
    bc[f * 9 + t] = pos;
}

// per-warp scratch of the node DP
struct NodeScratch {
    unsigned long long pk[kML][kML];  // [child slot][layer] packed best of each child
    double row[kML][kML];             // [low][layer] suffix minimum of the candidates of row `low`
    signed char row_at[kML][kML];     // [low][layer] the candidate's top layer
    double vcol[kML];                 // via costs of the node's column, layers 0..8
    double cost[kML];                 // the node's final cost per layer
    int win[kML];                     // winner low * 16 + top layer per layer, -1 none
};

constexpr double kNone = __builtin_huge_val();  // no candidate (every real candidate is below kInf)

// One net's DAG as the DP and the backtrace read it.  S = false: the batch
// arrays.  S = true: copied into shared memory at the start of the net (node
// positions decoded and packed as layer << 28 | x << 14 | y, child and
// parent-edge offsets, parents, child slots, level lists and level offsets,
// each node's via-cost column), with the packed child entries, the best
// paths, the chosen layers and the segment counts kept there too: only the
// offer records, the node costs and the segments go through L2.  Indices
// and values are the batch's in both forms.  Shared layout: u64
// packed[ms * 10], u64 best[ms * 10], double vcol[n * 8], then ints pos[n]
// coff[n+1] poff[n+1] lev[n] lo[n] scnt[n] par[m] slot[m] loff[levels + 1].
extern __shared__ __align__(16) unsigned long long s_dag[];
constexpr int kStageLevels = 64;  // levels of a staged net, at most
constexpr int kStageMaxSide = 1 << 14;  // staged positions hold x and y in 14 bits

struct NetLoc {
    int n0, e0, l0, c0;  // first node, parent edge, level offset and child slot
    int n, m, ms;        // nodes, parent edges, child slots
};

struct NodePos {
    int l, x, y;  // layer index (9: the Steiner layer) and GCell
};

// bytes of shared memory that a staged net of n nodes, m parent edges and ms
// child slots takes
__host__ __device__ constexpr size_t staged_bytes(int n, int m, int ms) {
    return 8 * (20 * (size_t)ms + 8 * (size_t)n) + 4 * (size_t)(6 * n + 2 + 2 * m + kStageLevels);
}

template <bool S>
struct Dag {
    const DagBatchDev &b;
    NetLoc L;
    int XY, Y;
    __device__ __forceinline__ int *ints() const { return reinterpret_cast<int *>(s_dag + 20 * L.ms + 8 * L.n); }
    __device__ __forceinline__ NodePos pos(int node) const {
        if (S) {
            const unsigned p = (unsigned)ints()[node - L.n0];
            return {(int)(p >> 28), (int)((p >> 14) & 0x3FFF), (int)(p & 0x3FFF)};
        }
        const int v = b.nodes[node], l = v / XY, q = v - l * XY, x = q / Y;
        return {l, x, q - x * Y};
    }
    __device__ __forceinline__ int coff(int node) const {
        return S ? ints()[L.n + node - L.n0] : b.child_off[node];
    }
    __device__ __forceinline__ int poff(int node) const {
        return S ? ints()[2 * L.n + 1 + node - L.n0] : b.par_off[node];
    }
    __device__ __forceinline__ int lev(int pos) const {
        return S ? ints()[3 * L.n + 2 + pos - L.n0] : b.level_nodes[pos];
    }
    __device__ __forceinline__ int *lo(int node) const {
        return S ? ints() + 4 * L.n + 2 + node - L.n0 : b.layer_out + node;
    }
    __device__ __forceinline__ int *scnt(int node) const {
        return S ? ints() + 5 * L.n + 2 + node - L.n0 : b.stage_cnt + node;
    }
    __device__ __forceinline__ int par(int e) const { return S ? ints()[6 * L.n + 2 + e - L.e0] : b.par[e]; }
    __device__ __forceinline__ int slot(int e) const {
        return S ? ints()[6 * L.n + 2 + L.m + e - L.e0] : b.child_slot[e];
    }
    __device__ __forceinline__ int loff(int d) const {
        return S ? ints()[6 * L.n + 2 + 2 * L.m + d] : b.level_off[L.l0 + d];
    }
    // packed entries and best paths of child slot `sl` (kML per slot)
    __device__ __forceinline__ unsigned long long *packed(int sl) const {
        return S ? s_dag + (sl - L.c0) * kML : b.packed + (int64_t)sl * kML;
    }
    __device__ __forceinline__ unsigned long long *best(int sl) const {
        return S ? s_dag + (L.ms + sl - L.c0) * kML : b.best_path + (int64_t)sl * kML;
    }
    // via costs of the node's column, layers 0..7 (staged nets)
    __device__ __forceinline__ const double *vcol(int node) const {
        return reinterpret_cast<const double *>(s_dag + 20 * L.ms) + (node - L.n0) * 8;
    }
};

// what one (parent edge, target layer t) pair needs besides the node's own
// costs: the parent's packed entry and, per source layer of t's parity
// (layer = 2 - t % 2 + 2q), the wire cost (layer == t, bit q of `wire`) or
// the precomputed mid-edge layer change cost (bit q of `change`; the
// reference skips it when it is not below INF).  The loads are only issued
// here: nothing reads their values until the offers are sent.
struct Offer {
    int64_t dst;
    double v[5];
    double mask;  // wire | change << 8, in the bits of a double (as stored)
};

template <bool S>
__device__ __forceinline__ void offer_load(const GridDev &g, const Dag<S> &D, int x, int y, int e, int t, Offer &o) {
    const int parent = D.par(e);
    const NodePos pp = D.pos(parent);
    const int px = pp.x, py = pp.y;
    const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
    const bool far = abs(x - px) + abs(y - py) > 4;
    o.dst = ((int64_t)D.coff(parent) + D.slot(e)) * kML + t;
    unsigned wire = 0, change = 0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int layer = 2 - (t & 1) + 2 * q;
        o.v[q] = kNone;
        if (layer >= kML) continue;
        const int dl = (layer & 1) ^ g.DIR;  // direction test of the reference, on 1-based layers
        if (dl == 1 && y != py) continue;
        if (dl == 0 && x != px) continue;
        if (t == layer) {
            o.v[q] = wire_cost(g, layer - 1, minx, maxx, miny, maxy);
            wire |= 1u << q;
        } else if (far) {
            o.v[q] = D.b.cost_edges[(int64_t)e * 81 + (layer - 1) * 9 + (t - 1)];
            change |= 1u << q;
        }
    }
    o.mask = __longlong_as_double((long long)(wire | change << 8));
}

// The offer records depend on no DP result: dag_offer_kernel computes them
// for every (parent edge, target layer) pair of the batch before the DP, at
// (e * 9 + t - 1) * kOfferRec in b.offers: v[0..4], then the mask.
constexpr int kOfferRec = 6;

__device__ __forceinline__ void offer_store(const DagBatchDev &b, int e, int t, const Offer &o) {
    double2 *r = reinterpret_cast<double2 *>(b.offers + ((int64_t)e * 9 + (t - 1)) * kOfferRec);
    r[0] = make_double2(o.v[0], o.v[1]);
    r[1] = make_double2(o.v[2], o.v[3]);
    r[2] = make_double2(o.v[4], o.mask);
}

template <bool S>
__device__ __forceinline__ void offer_fetch(const Dag<S> &D, int e, int t, Offer &o) {
    const double2 *r = reinterpret_cast<const double2 *>(D.b.offers + ((int64_t)e * 9 + (t - 1)) * kOfferRec);
    const double2 a = r[0], c = r[1], d = r[2];
    o.v[0] = a.x; o.v[1] = a.y; o.v[2] = c.x; o.v[3] = c.y; o.v[4] = d.x;
    o.mask = d.y;
    o.dst = ((int64_t)D.coff(D.par(e)) + D.slot(e)) * kML + t;
}

// the offer of pair (e, t): fetched, or computed without offer records
template <bool S>
__device__ __forceinline__ void offer_get(const GridDev &g, const Dag<S> &D, int x, int y, int e, int t, Offer &o) {
    if (D.b.offers)
        offer_fetch(D, e, t, o);
    else
        offer_load(g, D, x, y, e, t, o);
}

// one thread per (parent edge, target layer) pair of the batch
__global__ void __launch_bounds__(256) dag_offer_kernel(GridDev g, DagBatchDev b) {
    chain_begin();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)b.n_edges * 9) return;
    const int e = (int)(i / 9), t = 1 + (int)(i % 9);
    const Dag<false> D{b, NetLoc{}, g.X * g.Y, g.Y};
    const NodePos p = D.pos(b.edge_child[e]);
    Offer o;
    offer_load(g, D, p.x, p.y, e, t, o);
    offer_store(b, e, t, o);
}

// the minimum packed offer of the pair over its source layers, then atomicMin
// into the parent's entry (the minimum does not depend on the order)
template <bool S>
__device__ __forceinline__ void offer_send(const Dag<S> &D, const Offer &o, const double *cost, int node) {
    const int t = (int)(o.dst % kML);
    const unsigned mk = (unsigned)__double_as_longlong(o.mask), wire = mk & 0xff, change = mk >> 8;
    unsigned long long m = ~0ull;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int layer = 2 - (t & 1) + 2 * q;
        if (layer >= kML) continue;
        if (!((wire >> q) & 1) && !(((change >> q) & 1) && o.v[q] < kInf)) continue;
        const double c2 = cost[layer] + o.v[q];
        const int choice = t == layer ? 82 : (layer - 1) * 9 + (t - 1);
        const unsigned long long nv = pack((float)c2, node * 100 + choice);
        if (nv < m) m = nv;
    }
    if (m == ~0ull) return;
    if (S)
        atomicMin(s_dag + (o.dst - (int64_t)D.L.c0 * kML), m);
    else
        atomicMin(D.b.packed + o.dst, m);
}

// Lshape_route_node_layer_change_cuda for one node, computed by one warp.
//
// The reference walks low = 1..fixed_low; for each low it scans layer =
// low..9, keeping per child the first minimum of the packed costs over
// [low, layer] and the via cost of the column from low to layer, offers the
// candidate T(low, layer) = via + sum of the children's minima (for layer >=
// fixed_high, if below INF) to cost[layer] with a strict `<`, then copies
// cost[layer + 1] down to cost[layer] where strictly smaller, layer 8..low.
// Unrolling that order, cost[j] ends as the minimum of T(low, J) over
// low <= j <= J, and of equal candidates the one with the smallest low, then
// the smallest J, is the one that arrives first and stays; best[c][j] is then
// child c's first minimum over [low, J] of that winner.  The warp computes the
// 45 candidates row by row (lane = low, the same additions in the same order),
// the suffix minima of each row, and per layer the minimum over rows.
template <bool S>
__device__ void dp_node_warp(const GridDev &g, const Dag<S> &D, int node, int lane, NodeScratch &s) {
    const DagBatchDev &b = D.b;
    const NodePos np = D.pos(node);
    const int fixed_low = 1 + np.l;
    const int fixed_high = fixed_low == 10 ? 0 : fixed_low;
    const int x = np.x, y = np.y;
    const int cb = D.coff(node), cn = D.coff(node + 1) - cb;
    const int pb = D.poff(node), pn = D.poff(node + 1) - pb;
    __syncwarp();  // the previous node's scratch is no longer read
    // the children's packed entries (rows of kML) and the via costs of the
    // node's column: in shared memory where the net is staged, else loaded
    // here (past L1: the children's atomics landed in L2); every global load
    // of the node is issued before any is used
    const unsigned long long *pk;
    const double *vcol;
    Offer o;
    if (S) {
        pk = D.packed(cb);
        vcol = D.vcol(node);
        if (lane < pn * 9) offer_get(g, D, x, y, pb + lane / 9, 1 + lane % 9, o);
    } else {
        const unsigned long long *gp = b.packed + (int64_t)cb * kML;
        unsigned long long pkv[3];  // entries lane + 32 r of the cn * 9 <= 90
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const int i = lane + 32 * r;
            if (i < cn * 9) pkv[r] = __ldcg(gp + (i / 9) * kML + 1 + i % 9);
        }
        double vc = 0;
        if (lane < 8) vc = g.vcost[cell_at(g, lane, x, y)];
        if (lane < pn * 9) offer_get(g, D, x, y, pb + lane / 9, 1 + lane % 9, o);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const int i = lane + 32 * r;
            if (i < cn * 9) s.pk[i / 9][1 + i % 9] = pkv[r];
        }
        if (lane < 8) s.vcol[lane] = vc;
        __syncwarp();
        pk = &s.pk[0][0];
        vcol = s.vcol;
    }
    if (lane < 9) {
        // row `low`: T(low, J) = via(low, J) + the children's first minima
        // over [low, J], added child by child in child order (the
        // reference's order); J < low or low > fixed_low take no part
        const int low = lane + 1;
        const bool on = low <= fixed_low;
        double T[kML];
        double via = 0;
#pragma unroll
        for (int J = 1; J < kML; J++) {
            if (on && J > low) via += vcol[J - 2];
            T[J] = via;
        }
        for (int c = 0; c < cn; c++) {
            const unsigned long long *row = pk + c * kML;
            double m = kInf;
#pragma unroll
            for (int J = 1; J < kML; J++) {
                if (on && J >= low) {
                    const double cc = packed_cost(row[J]);
                    if (cc < m) m = cc;
                    T[J] += m;
                }
            }
        }
        double r = kNone;
        int rj = -1;
#pragma unroll
        for (int J = kML - 1; J >= 1; J--) {
            const bool cand = on && J >= low && J >= fixed_high && T[J] < kInf;
            if (cand && T[J] <= r) { r = T[J]; rj = J; }  // equal: the smaller top layer
            s.row[low][J] = r;
            s.row_at[low][J] = (signed char)rj;
        }
    }
    __syncwarp();
    double *cost = b.costs + (int64_t)node * kML;
    if (lane < 9) {
        const int j = lane + 1;
        double m = kNone;
        int wl = -1, wj = -1;
        for (int lo = 1; lo <= j; lo++) {
            const double r = s.row[lo][j];
            if (r < m) { m = r; wl = lo; wj = s.row_at[lo][j]; }  // equal: the smaller low
        }
        const double cj = wl > 0 ? m : kInf;
        s.cost[j] = cj;
        s.win[j] = wl > 0 ? wl * 16 + wj : -1;
        cost[j] = cj;
    } else if (lane == 9) {
        s.cost[0] = kInf;
        s.win[0] = -1;
        cost[0] = kInf;
    }
    __syncwarp();
    unsigned long long *best = D.best(cb);
    for (int i = lane; i < cn * kML; i += 32) {
        const int c = i / kML, j = i % kML;
        const int w = s.win[j];
        unsigned long long val = 0;
        if (w >= 0) {
            double m = kInf;
            for (int q = w >> 4; q <= (w & 15); q++) {
                const unsigned long long p = pk[c * kML + q];
                const double cc = packed_cost(p);
                if (cc < m) { m = cc; val = (unsigned long long)packed_id(p) * kML + q; }
            }
        }
        best[c * kML + j] = val;
    }
    for (int i = lane + 32; i < pn * 9; i += 32) {
        Offer o2;
        offer_get(g, D, x, y, pb + i / 9, 1 + i % 9, o2);
        offer_send(D, o2, s.cost, node);
    }
    if (lane < pn * 9) offer_send(D, o, s.cost, node);
}

template <bool S>
__device__ __forceinline__ void stage2(const Dag<S> &D, int node, int a, int c, int *err) {
    int *cnt = D.scnt(node);
    const int k = *cnt;
    if (k + 2 > 8) { set_error(err, ERR_CAPACITY); return; }
    D.b.stage[(int64_t)node * 8 + k] = a;
    D.b.stage[(int64_t)node * 8 + k + 1] = c;
    *cnt = k + 2;
}

// get_routing_tree_layer_change_cuda for one node
template <bool S>
__device__ void trace_node(const GridDev &g, const Dag<S> &D, int node, int stamp) {
    const DagBatchDev &b = D.b;
    const int X = g.X, Y = g.Y, XY = X * Y;
    const int pb = D.poff(node), pn = D.poff(node + 1) - pb;
    const NodePos np = D.pos(node);
    const int l = np.l, cx = np.x, cy = np.y;
    const unsigned long long *best = D.best(D.coff(node));
    int *lo = D.lo(node);
    if (pn == 0) {
        int ml = 0;
        double mc = b.costs[(int64_t)node * kML];
        for (int layer = 1; layer < kML; layer++)
            if (b.costs[(int64_t)node * kML + layer] < mc) { mc = b.costs[(int64_t)node * kML + layer]; ml = layer; }
        *lo = ml;
    } else {
        int par_layer = -1, par_idx = -1, par_seq = -1;
        for (int pi = 0; pi < pn; pi++) {
            const int e = pb + pi;
            const int pnode = D.par(e);
            if (*D.lo(pnode) > 0) {
                par_idx = pnode;
                par_seq = pi;
                par_layer = *D.lo(pnode);
                const int slot = D.slot(pb + par_seq);
                const unsigned long long path = D.best(D.coff(par_idx) + slot)[par_layer];
                const unsigned long long cid = path / kML / 100;
                const unsigned long long ch = (path / kML) % 100;
                if (cid == (unsigned long long)node) {
                    *lo = ch == 82 ? (int)(path % kML) : (int)(ch / 9 + 1);
                    const NodePos pp = D.pos(par_idx);
                    const int px = pp.x, py = pp.y;
                    const int L1 = *lo - 1;
                    if (px == cx && cy != py) {
                        if (ch == 82) {
                            add_wire(g, L1, px, px, min(py, cy), max(py, cy), stamp);
                            stage2(D, node, L1 * XY + px * Y + min(py, cy), L1 * XY + px * Y + max(py, cy), g.err);
                        } else {
                            const int fl = (int)(ch / 9), tl = (int)(ch % 9);
                            const int cp = b.best_change[(int64_t)e * 81 + fl * 9 + tl];
                            if (cp <= min(cy, py) || cp >= max(cy, py)) { set_error(g.err, ERR_STATE); return; }
                            add_wire(g, fl, cx, cx, min(cy, cp), max(cy, cp), stamp);
                            add_wire(g, tl, cx, cx, min(py, cp), max(py, cp), stamp);
                            stage2(D, node, fl * XY + cx * Y + min(cy, cp), fl * XY + cx * Y + max(cy, cp), g.err);
                            stage2(D, node, min(fl, tl) * XY + cx * Y + cp, max(fl, tl) * XY + cx * Y + cp, g.err);
                            stage2(D, node, tl * XY + cx * Y + min(py, cp), tl * XY + cx * Y + max(py, cp), g.err);
                        }
                    } else if (py == cy && cx != px) {
                        if (ch == 82) {
                            add_wire(g, L1, min(px, cx), max(px, cx), py, py, stamp);
                            stage2(D, node, L1 * XY + min(px, cx) * Y + py, L1 * XY + max(px, cx) * Y + py, g.err);
                        } else {
                            const int fl = (int)(ch / 9), tl = (int)(ch % 9);
                            const int cp = b.best_change[(int64_t)e * 81 + fl * 9 + tl];
                            if (cp <= min(cx, px) || cp >= max(cx, px)) { set_error(g.err, ERR_STATE); return; }
                            add_wire(g, fl, min(cx, cp), max(cx, cp), cy, cy, stamp);
                            add_wire(g, tl, min(px, cp), max(px, cp), cy, cy, stamp);
                            stage2(D, node, fl * XY + min(cx, cp) * Y + cy, fl * XY + max(cx, cp) * Y + cy, g.err);
                            stage2(D, node, min(fl, tl) * XY + cp * Y + cy, max(fl, tl) * XY + cp * Y + cy, g.err);
                            stage2(D, node, tl * XY + min(px, cp) * Y + cy, tl * XY + max(px, cp) * Y + cy, g.err);
                        }
                    }
                    break;
                } else {
                    *lo = -1;
                }
            }
        }
        if (par_layer == -1) { *lo = -1; return; }
        const int slot = D.slot(pb + par_seq);
        const unsigned long long path = D.best(D.coff(par_idx) + slot)[par_layer];
        if (path / kML / 100 != (unsigned long long)node) { *lo = -1; return; }
    }
    const int cn = D.coff(node + 1) - D.coff(node);
    const int lon = *lo;
    int mnl = l + 1;
    int mxl = (l + 1) == kML ? 1 : mnl;
    mnl = min(mnl, lon);
    mxl = max(mxl, lon);
    for (int c = 0; c < cn; c++) {
        const int lc = (int)(best[c * kML + lon] % kML);
        mnl = min(lc, mnl);
        mxl = max(lc, mxl);
    }
    if (mnl < mxl) stage2(D, node, (mnl - 1) * XY + cx * Y + cy, (mxl - 1) * XY + cx * Y + cy, g.err);
}

// route record of net k in DAG node order, written by one warp
template <bool S>
__device__ void compact_net(const GridDev &g, const Dag<S> &D, int k, int lane) {
    const DagBatchDev &b = D.b;
    const int net = b.net_ids[k];
    int *r = b.routes + b.route_off[net];
    const int cap = b.route_cap[net];
    const int n0 = D.L.n0, n1 = D.L.n0 + D.L.n;
    int base = 1;
    for (int c0 = n0; c0 < n1; c0 += 32) {
        const int node = c0 + lane;
        const int cnt = node < n1 ? *D.scnt(node) : 0;
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const int at = base + inc - cnt;
        if (cnt && at + cnt <= cap)
            for (int j = 0; j < cnt; j++) r[at + j] = b.stage[(int64_t)node * 8 + j];
        else if (cnt)
            set_error(g.err, ERR_CAPACITY);
        base += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) r[0] = base <= cap ? base : 1;
}

// one net: initialisation (and the copy into shared memory when staged), DP
// levels deepest first, trace levels root first, compaction
template <int W, bool S>
__device__ void route_net(const GridDev &g, const DagBatchDev &b, int k, const NetLoc &L, int nl, int stamp,
                          NodeScratch *scr) {
    constexpr int kThreadsW = 32 * W;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Dag<S> D{b, L, g.X * g.Y, g.Y};
    const int n0 = L.n0, n1 = L.n0 + L.n;
    if (S) {
        const int n = L.n, m = L.m, XY = g.X * g.Y;
        for (int i = tid; i < L.ms * kML; i += kThreadsW) s_dag[i] = kInitPacked;
        double *vcol = reinterpret_cast<double *>(s_dag + 20 * L.ms);
        int *I = D.ints();
        for (int i = tid; i < n; i += kThreadsW) {
            const int v = b.nodes[n0 + i], l = v / XY, q = v - l * XY, x = q / g.Y, y = q - x * g.Y;
            I[i] = (l << 28) | (x << 14) | y;
            I[3 * n + 2 + i] = b.level_nodes[n0 + i];
            I[4 * n + 2 + i] = -1;
            I[5 * n + 2 + i] = 0;
#pragma unroll
            for (int c = 0; c < kML - 2; c++) vcol[i * 8 + c] = g.vcost[cell_at(g, c, x, y)];
        }
        for (int i = tid; i <= n; i += kThreadsW) {
            I[n + i] = b.child_off[n0 + i];
            I[2 * n + 1 + i] = b.par_off[n0 + i];
        }
        for (int j = tid; j < m; j += kThreadsW) {
            I[6 * n + 2 + j] = b.par[L.e0 + j];
            I[6 * n + 2 + m + j] = b.child_slot[L.e0 + j];
        }
        for (int d = tid; d <= nl; d += kThreadsW) I[6 * n + 2 + 2 * m + d] = b.level_off[L.l0 + d];
    } else {
        const int64_t s0 = (int64_t)L.c0 * kML, s1 = (int64_t)(L.c0 + L.ms) * kML;
        for (int64_t i = s0 + tid; i < s1; i += kThreadsW) b.packed[i] = kInitPacked;
        for (int v = n0 + tid; v < n1; v += kThreadsW) {
            b.layer_out[v] = -1;
            b.stage_cnt[v] = 0;
        }
    }
    __syncthreads();
    for (int d = nl - 1; d >= 0; d--) {
        const int a = D.loff(d), e = D.loff(d + 1);
        for (int s = a + warp; s < e; s += W) dp_node_warp(g, D, D.lev(s), lane, scr[warp]);
        __syncthreads();
    }
    for (int d = 0; d < nl; d++) {
        const int a = D.loff(d), e = D.loff(d + 1);
        for (int s = a + tid; s < e; s += kThreadsW) trace_node(g, D, D.lev(s), stamp);
        __syncthreads();
    }
    if (warp == 0) compact_net(g, D, k, lane);
}

// one CTA of W warps per net.  Sizes: 0 every net, 1 nets of at most
// split_at nodes, 2 the larger ones.  A net of at most cap_n nodes and
// kStageLevels - 1 levels whose staged_bytes fit the launch's dynamic shared
// memory (smem) is staged there.  At most 80 registers a thread: 12 CTAs of
// 2 warps, 3 of 8 warps, or one of 16 warps beside one of 8 per SM.
template <int W, int Sizes>
__global__ void __maxnreg__(80) dag_net_kernel(GridDev g, DagBatchDev b, int stamp, int cap_n, int smem,
                                               int split_at) {
    chain_begin();
    __shared__ NodeScratch scr[W];
    for (int k = blockIdx.x; k < b.n_nets; k += gridDim.x) {
        const int n0 = b.net_node_off[k], n1 = b.net_node_off[k + 1];
        if ((Sizes == 1 && n1 - n0 > split_at) || (Sizes == 2 && n1 - n0 <= split_at)) continue;
        const int l0 = b.net_level_off[k], nl = b.net_level_off[k + 1] - l0 - 1;
        const int e0 = b.par_off[n0], c0 = b.child_off[n0];
        const NetLoc L{n0, e0, l0, c0, n1 - n0, b.par_off[n1] - e0, b.child_off[n1] - c0};
        if (L.n <= cap_n && nl < kStageLevels && staged_bytes(L.n, L.m, L.ms) <= (size_t)smem)
            route_net<W, true>(g, b, k, L, nl, stamp, scr);
        else
            route_net<W, false>(g, b, k, L, nl, stamp, scr);
        __syncthreads();
    }
}

}  // namespace

void dag_levels(int n, const int *node_off, const int *depth, std::vector<int> &level_nodes,
                std::vector<int> &level_off, std::vector<int> &net_level_off) {
    level_nodes.resize(node_off[n] - node_off[0]);
    level_off.clear();
    net_level_off.assign(1, 0);
    std::vector<int> cnt;
    for (int k = 0; k < n; k++) {
        const int a = node_off[k], e = node_off[k + 1];
        int D = 0;
        for (int v = a; v < e; v++) D = std::max(D, depth[v] + 1);
        cnt.assign(D + 1, 0);
        for (int v = a; v < e; v++) cnt[depth[v] + 1]++;
        cnt[0] = a - node_off[0];
        for (int d = 0; d < D; d++) cnt[d + 1] += cnt[d];
        level_off.insert(level_off.end(), cnt.begin(), cnt.end());
        for (int v = a; v < e; v++) level_nodes[cnt[depth[v]]++] = v;
        net_level_off.push_back((int)level_off.size());
    }
}

int launch_dag_route(const GridDev &g, const DagBatchDev &b, int stamp, cudaStream_t s, cudaStream_t aux,
                     cudaEvent_t fork, cudaEvent_t join, int split_nets, int stage_nodes) {
    if (b.n_nodes <= 0 || b.n_nets <= 0) return 0;
    int launches = 0;
    if (b.n_edges > 0) {
        launch_chained(dag_edge_cost_kernel, dim3((int)((b.n_edges + kEdgeWarps - 1) / kEdgeWarps)),
                       dim3(32 * kEdgeWarps), 0, s, g, b);
        launches++;
        if (b.offers) {
            launch_chained(dag_offer_kernel, dim3((int)(((int64_t)b.n_edges * 9 + 255) / 256)), dim3(256), 0, s, g, b);
            launches++;
        }
    }
    // Staging: none without room for offer records or where positions do not
    // fit their packed form.  The shared memory of a launch fits the largest
    // net of its size class (rounded up, so that few distinct sizes occur),
    // within what a CTA can have; nets that do not fit run unstaged.
    const int cap_n = b.offers && g.X <= kStageMaxSide && g.Y <= kStageMaxSide ? std::max(0, stage_nodes) : 0;
    auto fit = [&](int n, int m, int warps) -> int {
        if (!cap_n || n <= 0) return 0;
        const size_t room = (size_t)dag_solo_smem_limit() - sizeof(NodeScratch) * warps;
        const int nn = (std::min(n, cap_n) + 31) / 32 * 32, mm = (std::min(m, 2 * nn) + 63) / 64 * 64;
        return (int)std::min(staged_bytes(nn, mm, mm), room);
    };
    const int mx_n = b.max_net_nodes > 0 ? b.max_net_nodes : cap_n;
    const int mx_m = b.max_net_edges > 0 ? b.max_net_edges : 2 * mx_n;
    const bool many = aux && b.n_nets >= split_nets;
    const bool two = aux && !many && mx_n > kSmallStageNodes && cap_n > 0;
    if (!many && !two) {
        const int smem = fit(mx_n, mx_m, kDagWarps);
        kernel_setup((const void *)dag_net_kernel<kDagWarps, 0>, kDagThreads, smem);
        launch_chained(dag_net_kernel<kDagWarps, 0>, dim3(b.n_nets), dim3(kDagThreads), (size_t)smem, s, g, b, stamp,
                       cap_n, smem, 0);
        return launches + 1;
    }
    // two launches over the batch, each taking the nets of its size class
    // (the nets of a batch share no state): the larger nets' CTAs on the side
    // stream, beside the smaller nets' CTAs, whose shared memory is sized for
    // their class
    const int split_at = many ? kSmallNodes : kSmallStageNodes;
    const int small_w = many ? kSmallWarps : kDagWarps;
    const int smem_small = fit(std::min(mx_n, split_at), std::min(mx_m, 2 * split_at), small_w);
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(aux, fork, 0);
    if (many) {
        const int smem_large = fit(mx_n, mx_m, kDagWarps);
        kernel_setup((const void *)dag_net_kernel<kDagWarps, 2>, kDagThreads, smem_large);
        dag_net_kernel<kDagWarps, 2><<<b.n_nets, kDagThreads, smem_large, aux>>>(g, b, stamp, cap_n, smem_large,
                                                                                split_at);
    } else {
        // the larger DAGs bound the batch: their CTAs take 16 warps, so that
        // their wide levels take fewer rounds
        const int smem_large = fit(mx_n, mx_m, kBigWarps);
        kernel_setup((const void *)dag_net_kernel<kBigWarps, 2>, 32 * kBigWarps, smem_large);
        dag_net_kernel<kBigWarps, 2><<<b.n_nets, 32 * kBigWarps, smem_large, aux>>>(g, b, stamp, cap_n, smem_large,
                                                                                   split_at);
    }
    if (many) {
        // a batch of many nets: the DAGs of at most kSmallNodes nodes in
        // 2-warp CTAs, so that more of them are in flight
        kernel_setup((const void *)dag_net_kernel<kSmallWarps, 1>, 32 * kSmallWarps, smem_small);
        dag_net_kernel<kSmallWarps, 1><<<b.n_nets, 32 * kSmallWarps, smem_small, s>>>(g, b, stamp, cap_n, smem_small,
                                                                                      split_at);
    } else {
        kernel_setup((const void *)dag_net_kernel<kDagWarps, 1>, kDagThreads, smem_small);
        dag_net_kernel<kDagWarps, 1><<<b.n_nets, kDagThreads, smem_small, s>>>(g, b, stamp, cap_n, smem_small,
                                                                              split_at);
    }
    cudaEventRecord(join, aux);
    cudaStreamWaitEvent(s, join, 0);
    return launches + 2;
}

}  // namespace igr
