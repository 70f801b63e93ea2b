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

// what one (parent edge, target layer t) pair needs besides the node's own
// costs: the parent's packed entry and, per source layer of t's parity
// (layer = 2 - t % 2 + 2q), the wire cost (layer == t) or the precomputed
// mid-edge layer change cost, kNone where the reference skips the layer
struct Offer {
    int64_t dst;
    double v[5];
};

__device__ __forceinline__ void offer_load(const GridDev &g, const DagBatchDev &b, int node, int x, int y, int e,
                                           int t, Offer &o) {
    const int parent = b.par[e];
    const int pv = b.nodes[parent];
    const int px = pv / g.Y % g.X, py = pv % g.Y;
    const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
    const bool far = abs(x - px) + abs(y - py) > 4;
    o.dst = ((int64_t)b.child_off[parent] + b.child_slot[e]) * kML + t;
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
        } else if (far) {
            const double ce = b.cost_edges[(int64_t)e * 81 + (layer - 1) * 9 + (t - 1)];
            if (ce < kInf) o.v[q] = ce;
        }
    }
}

// the minimum packed offer of the pair over its source layers, then atomicMin
// into the parent's entry (the minimum does not depend on the order)
__device__ __forceinline__ void offer_send(const DagBatchDev &b, const Offer &o, const double *cost, int node) {
    const int t = (int)(o.dst % kML);
    unsigned long long m = ~0ull;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int layer = 2 - (t & 1) + 2 * q;
        if (layer >= kML || !(o.v[q] < kNone)) continue;
        const double c2 = cost[layer] + o.v[q];
        const int choice = t == layer ? 82 : (layer - 1) * 9 + (t - 1);
        const unsigned long long nv = pack((float)c2, node * 100 + choice);
        if (nv < m) m = nv;
    }
    if (m != ~0ull) atomicMin(b.packed + o.dst, m);
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
__device__ void dp_node_warp(const GridDev &g, const DagBatchDev &b, int node, int lane, NodeScratch &s) {
    const int X = g.X, Y = g.Y, XY = X * Y;
    const int v = b.nodes[node];
    const int fixed_low = 1 + v / XY;
    const int fixed_high = fixed_low == 10 ? 0 : fixed_low;
    const int x = v / Y % X, y = v % Y;
    const int cb = b.child_off[node], cn = b.child_off[node + 1] - cb;
    __syncwarp();  // the previous node's scratch is no longer read
    {
        // the children's atomics landed in L2: read past L1
        const unsigned long long *pk = b.packed + (int64_t)cb * kML;
        for (int i = lane; i < cn * 9; i += 32) {
            const int c = i / 9, layer = 1 + i % 9;
            s.pk[c][layer] = __ldcg(pk + c * kML + layer);
        }
        if (lane < 8) s.vcol[lane] = g.vcost[cell_at(g, lane, x, y)];
    }
    // the parent-side inputs do not depend on the DP: issue their loads now
    const int pb = b.par_off[node], pn = b.par_off[node + 1] - pb;
    Offer o;
    if (lane < pn * 9) offer_load(g, b, node, x, y, pb + lane / 9, 1 + lane % 9, o);
    __syncwarp();
    if (lane < 9) {
        const int low = lane + 1;
        double T[kML];
        double minc[kML];
#pragma unroll
        for (int c = 0; c < kML; c++) minc[c] = kInf;
        double via = 0;
#pragma unroll
        for (int J = 1; J < kML; J++) {
            T[J] = kNone;
            if (J >= low && low <= fixed_low) {
                if (J > low) via += s.vcol[J - 2];
                double t = via;
#pragma unroll
                for (int c = 0; c < kML; c++) {
                    if (c < cn) {
                        const double cc = packed_cost(s.pk[c][J]);
                        if (cc < minc[c]) minc[c] = cc;
                        t += minc[c];
                    }
                }
                if (J >= fixed_high && t < kInf) T[J] = t;
            }
        }
        double r = kNone;
        int rj = -1;
#pragma unroll
        for (int J = kML - 1; J >= 1; J--) {
            if (T[J] < kNone && T[J] <= r) { r = T[J]; rj = J; }  // equal: the smaller top layer
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
    unsigned long long *best = b.best_path + (int64_t)cb * kML;
    for (int i = lane; i < cn * kML; i += 32) {
        const int c = i / kML, j = i % kML;
        const int w = s.win[j];
        unsigned long long val = 0;
        if (w >= 0) {
            double m = kInf;
            for (int q = w >> 4; q <= (w & 15); q++) {
                const unsigned long long p = s.pk[c][q];
                const double cc = packed_cost(p);
                if (cc < m) { m = cc; val = (unsigned long long)packed_id(p) * kML + q; }
            }
        }
        best[c * kML + j] = val;
    }
    for (int i = lane + 32; i < pn * 9; i += 32) {
        Offer o2;
        offer_load(g, b, node, x, y, pb + i / 9, 1 + i % 9, o2);
        offer_send(b, o2, s.cost, node);
    }
    if (lane < pn * 9) offer_send(b, o, s.cost, node);
}

__device__ __forceinline__ void stage2(const DagBatchDev &b, int node, int a, int c, int *err) {
    int k = b.stage_cnt[node];
    if (k + 2 > 8) { set_error(err, ERR_CAPACITY); return; }
    b.stage[(int64_t)node * 8 + k] = a;
    b.stage[(int64_t)node * 8 + k + 1] = c;
    b.stage_cnt[node] = k + 2;
}

// get_routing_tree_layer_change_cuda for one node
__device__ void trace_node(const GridDev &g, const DagBatchDev &b, int node, int stamp) {
    const int X = g.X, Y = g.Y, XY = X * Y;
    const int pb = b.par_off[node], pn = b.par_off[node + 1] - pb;
    const int v = b.nodes[node];
    const int l = v / XY, cx = v / Y % X, cy = v % Y;
    const unsigned long long *best = b.best_path + (int64_t)b.child_off[node] * kML;
    int *lo = b.layer_out;
    if (pn == 0) {
        int ml = 0;
        double mc = b.costs[(int64_t)node * kML];
        for (int layer = 1; layer < kML; layer++)
            if (b.costs[(int64_t)node * kML + layer] < mc) { mc = b.costs[(int64_t)node * kML + layer]; ml = layer; }
        lo[node] = ml;
    } else {
        int par_layer = -1, par_idx = -1, par_seq = -1;
        for (int pi = 0; pi < pn; pi++) {
            const int e = pb + pi;
            const int pnode = b.par[e];
            if (lo[pnode] > 0) {
                par_idx = pnode;
                par_seq = pi;
                par_layer = lo[pnode];
                const int slot = b.child_slot[pb + par_seq];
                const unsigned long long path = b.best_path[(int64_t)b.child_off[par_idx] * kML + slot * kML + par_layer];
                const unsigned long long cid = path / kML / 100;
                const unsigned long long ch = (path / kML) % 100;
                if (cid == (unsigned long long)node) {
                    lo[node] = ch == 82 ? (int)(path % kML) : (int)(ch / 9 + 1);
                    const int pv = b.nodes[par_idx];
                    const int px = pv / Y % X, py = pv % Y;
                    const int L1 = lo[node] - 1;
                    if (px == cx && cy != py) {
                        if (ch == 82) {
                            add_wire(g, L1, px, px, min(py, cy), max(py, cy), stamp);
                            stage2(b, node, L1 * XY + px * Y + min(py, cy), L1 * XY + px * Y + max(py, cy), g.err);
                        } else {
                            const int fl = (int)(ch / 9), tl = (int)(ch % 9);
                            const int cp = b.best_change[(int64_t)e * 81 + fl * 9 + tl];
                            if (cp <= min(cy, py) || cp >= max(cy, py)) { set_error(g.err, ERR_STATE); return; }
                            add_wire(g, fl, cx, cx, min(cy, cp), max(cy, cp), stamp);
                            add_wire(g, tl, cx, cx, min(py, cp), max(py, cp), stamp);
                            stage2(b, node, fl * XY + cx * Y + min(cy, cp), fl * XY + cx * Y + max(cy, cp), g.err);
                            stage2(b, node, min(fl, tl) * XY + cx * Y + cp, max(fl, tl) * XY + cx * Y + cp, g.err);
                            stage2(b, node, tl * XY + cx * Y + min(py, cp), tl * XY + cx * Y + max(py, cp), g.err);
                        }
                    } else if (py == cy && cx != px) {
                        if (ch == 82) {
                            add_wire(g, L1, min(px, cx), max(px, cx), py, py, stamp);
                            stage2(b, node, L1 * XY + min(px, cx) * Y + py, L1 * XY + max(px, cx) * Y + py, g.err);
                        } else {
                            const int fl = (int)(ch / 9), tl = (int)(ch % 9);
                            const int cp = b.best_change[(int64_t)e * 81 + fl * 9 + tl];
                            if (cp <= min(cx, px) || cp >= max(cx, px)) { set_error(g.err, ERR_STATE); return; }
                            add_wire(g, fl, min(cx, cp), max(cx, cp), cy, cy, stamp);
                            add_wire(g, tl, min(px, cp), max(px, cp), cy, cy, stamp);
                            stage2(b, node, fl * XY + min(cx, cp) * Y + cy, fl * XY + max(cx, cp) * Y + cy, g.err);
                            stage2(b, node, min(fl, tl) * XY + cp * Y + cy, max(fl, tl) * XY + cp * Y + cy, g.err);
                            stage2(b, node, tl * XY + min(px, cp) * Y + cy, tl * XY + max(px, cp) * Y + cy, g.err);
                        }
                    }
                    break;
                } else {
                    lo[node] = -1;
                }
            }
        }
        if (par_layer == -1) { lo[node] = -1; return; }
        const int slot = b.child_slot[pb + par_seq];
        const unsigned long long path = b.best_path[(int64_t)b.child_off[par_idx] * kML + slot * kML + par_layer];
        if (path / kML / 100 != (unsigned long long)node) { lo[node] = -1; return; }
    }
    const int cn = b.child_off[node + 1] - b.child_off[node];
    int mnl = l + 1;
    int mxl = (l + 1) == kML ? 1 : mnl;
    mnl = min(mnl, lo[node]);
    mxl = max(mxl, lo[node]);
    for (int c = 0; c < cn; c++) {
        const int lc = (int)(best[c * kML + lo[node]] % kML);
        mnl = min(lc, mnl);
        mxl = max(lc, mxl);
    }
    if (mnl < mxl) stage2(b, node, (mnl - 1) * XY + cx * Y + cy, (mxl - 1) * XY + cx * Y + cy, g.err);
}

// route record of net k in DAG node order, written by one warp
__device__ void compact_net(const GridDev &g, const DagBatchDev &b, int k, int lane) {
    const int net = b.net_ids[k];
    int *r = b.routes + b.route_off[net];
    const int cap = b.route_cap[net];
    const int n0 = b.net_node_off[k], n1 = b.net_node_off[k + 1];
    int base = 1;
    for (int c0 = n0; c0 < n1; c0 += 32) {
        const int node = c0 + lane;
        const int cnt = node < n1 ? b.stage_cnt[node] : 0;
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

// one CTA of W warps per net: initialisation, DP levels deepest first, trace
// levels root first, compaction.  Sizes: 0 every net, 1 nets of at most
// kSmallNodes nodes, 2 the larger ones (small DAGs have narrow levels, so a
// 2-warp CTA leaves fewer warps waiting at the level barriers and more CTAs
// fit an SM)
template <int W, int Sizes>
__global__ void __launch_bounds__(32 * W) dag_net_kernel(GridDev g, DagBatchDev b, int stamp) {
    chain_begin();
    constexpr int kThreadsW = 32 * W;
    __shared__ NodeScratch scr[W];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int k = blockIdx.x; k < b.n_nets; k += gridDim.x) {
        const int n0 = b.net_node_off[k], n1 = b.net_node_off[k + 1];
        if ((Sizes == 1 && n1 - n0 > kSmallNodes) || (Sizes == 2 && n1 - n0 <= kSmallNodes)) continue;
        const int64_t s0 = (int64_t)b.child_off[n0] * kML, s1 = (int64_t)b.child_off[n1] * kML;
        for (int64_t i = s0 + tid; i < s1; i += kThreadsW) b.packed[i] = kInitPacked;
        for (int v = n0 + tid; v < n1; v += kThreadsW) {
            b.layer_out[v] = -1;
            b.stage_cnt[v] = 0;
        }
        __syncthreads();
        const int l0 = b.net_level_off[k], nl = b.net_level_off[k + 1] - l0 - 1;
        for (int d = nl - 1; d >= 0; d--) {
            const int a = b.level_off[l0 + d], e = b.level_off[l0 + d + 1];
            for (int s = a + warp; s < e; s += W) dp_node_warp(g, b, b.level_nodes[s], lane, scr[warp]);
            __syncthreads();
        }
        for (int d = 0; d < nl; d++) {
            const int a = b.level_off[l0 + d], e = b.level_off[l0 + d + 1];
            for (int s = a + tid; s < e; s += kThreadsW) trace_node(g, b, b.level_nodes[s], stamp);
            __syncthreads();
        }
        if (warp == 0) compact_net(g, b, k, lane);
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
                     cudaEvent_t fork, cudaEvent_t join, int split_nets) {
    if (b.n_nodes <= 0 || b.n_nets <= 0) return 0;
    int launches = 0;
    if (b.n_edges > 0) {
        launch_chained(dag_edge_cost_kernel, dim3((int)((b.n_edges + kEdgeWarps - 1) / kEdgeWarps)),
                       dim3(32 * kEdgeWarps), 0, s, g, b);
        launches++;
    }
    if (!aux || b.n_nets < split_nets) {
        launch_chained(dag_net_kernel<kDagWarps, 0>, dim3(b.n_nets), dim3(kDagThreads), 0, s, g, b, stamp);
        return launches + 1;
    }
    // a batch of many nets: the large nets' CTAs on the side stream, beside
    // the small nets' 2-warp CTAs (the nets of a batch share no state); a
    // smaller batch is bound by its largest net and gains nothing from it
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(aux, fork, 0);
    dag_net_kernel<kDagWarps, 2><<<b.n_nets, kDagThreads, 0, aux>>>(g, b, stamp);
    dag_net_kernel<kSmallWarps, 1><<<b.n_nets, 32 * kSmallWarps, 0, s>>>(g, b, stamp);
    cudaEventRecord(join, aux);
    cudaStreamWaitEvent(s, join, 0);
    return launches + 2;
}

}  // namespace igr
