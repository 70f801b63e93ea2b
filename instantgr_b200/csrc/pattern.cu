// Phase-1 pattern routing: layer-assignment DP over each net's Steiner tree
// with straight and L-shaped edges, then backtrace, route emission and demand
// difference-array updates.
//
// Restates Lshape_route_cuda (src/Lshape_route.hpp:9-153).  The reference runs
// one thread per net with 81-entry f64 tables per node in global memory (928
// bytes of stack per thread), and every tree edge waits on its own gathers.
// Here a group of G lanes (G = 16 or 32) owns a net:
//   1. every cost the net needs that depends only on geometry (via-stack
//      columns of its nodes, the wire cost of each leg on each layer, the via
//      columns at both corners of each bent edge) is gathered up front, all
//      lanes in parallel, into shared memory;
//   2. the edges are then processed bottom-up from shared memory only: the
//      lanes work on the nine layers, the nine target layers of a bend (each
//      looping over the 4-5 bend layers of opposite parity in the reference's
//      order), the nine range rows (with the reference's <= rule) and the
//      accumulation into the parent (in the reference's order of additions);
//   3. one lane fixes every node's layer range in preorder (shared memory
//      only); then all lanes emit the route record and write the difference
//      array, each node's segments placed by a prefix sum over the nodes.
// Nets are taken from a per-batch queue in the order given (largest first),
// so the long nets of a batch start early.  The 45 valid layer ranges of a
// node live in shared memory (global scratch for nets of more than kNodeTile
// nodes).  For the same cost map the chosen layers, routes and demand are
// bit-identical to the reference's.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kL = kRouteL;                  // 9 routing layers
constexpr int kR = 45;                       // layer ranges minl <= maxl
constexpr int kPF = 36;                      // prefetched doubles per edge
constexpr int kCol = kL - 1;                 // via column per node: vcost of layers 0..7

__host__ __device__ constexpr int tri(int a, int b) { return a * 9 - a * (a - 1) / 2 + (b - a); }

template <int T>
struct GroupSmem {
    double dist[T * kR];
    double pf[2 * kPF];  // geometry-only costs of the current and the next edge
    float col[T * kCol];
    short from[T * kR];  // backtrace code of each range: cf * 81 + child layer * 9 + parent layer
    int lr[T];
    int nx[T], ny[T], nl[T], np[T];  // decoded node position and parent
    double costc[kL], diag[kL];
    int cf[kL], pdiag[kL];
};

__device__ __forceinline__ double wire_cost(const GridDev &g, int l, int xa, int xb, int ya, int yb) {
    // presum[IDX(l, xmax, ymax)] - presum[IDX(l, xmin, ymin)]  (graph.hpp:19-21)
    return g.presum[cell_at(g, l, xb, yb)] - g.presum[cell_at(g, l, xa, ya)];
}

// Geometry-only cost j of the edge from (x, y) to its parent (px, py), 0 when
// unused: [0,9) child leg (bent) or wire (straight) per layer, [9,18) parent
// leg, [18,27) via column at (x, py), [27,36) via column at (px, y).
__device__ __forceinline__ double edge_value(const GridDev &g, int x, int y, int px, int py, int j) {
    const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
    const bool straight = (x == px || y == py);
    if (j < kL) {
        const int l = j;
        if (straight) {
            const int dl = layer_dir(g, l);
            if (!((dl == 0 && y != py) || (dl == 1 && x != px))) return wire_cost(g, l, minx, maxx, miny, maxy);
            return 0.0;
        }
        return layer_dir(g, l) ? wire_cost(g, l, x, x, miny, maxy) : wire_cost(g, l, minx, maxx, y, y);
    }
    if (straight) return 0.0;
    if (j < 2 * kL) {
        const int l = j - kL;
        return layer_dir(g, l) ? wire_cost(g, l, px, px, miny, maxy) : wire_cost(g, l, minx, maxx, py, py);
    }
    if (j < 3 * kL) return (double)g.vcost[cell_at(g, j - 2 * kL, x, py)];
    return (double)g.vcost[cell_at(g, j - 3 * kL, px, y)];
}

__device__ __forceinline__ void add_wire(const GridDev &g, const int *layer_first, int l, int xa, int xb, int ya,
                                         int yb, int stamp) {
    // atomic_add_unit_demand_wire_segment (graph.hpp:105-117), K = 1
    atomicAdd(&g.pre[cell_at(g, l, xa, ya)], 1);
    if (xa == xb) {
        atomicAdd(&g.pre[cell_at(g, l, xa, yb)], -1);
        g.stamp[cell_at(g, l, xa, yb)] = stamp;
    }
    if (ya == yb) {
        atomicAdd(&g.pre[cell_at(g, l, xb, ya)], -1);
        g.stamp[cell_at(g, l, xb, ya)] = stamp;
    }
    g.dirty_commit[track_of(g, l, xa, ya, layer_first)] = 1;
}

// Via crossings of a via span [lo, hi) at (x, y) for the fused batch commit.
__device__ __forceinline__ void count_vias(const GridDev &g, int *vcnt, const int *layer_first, int lo, int hi, int x,
                                           int y) {
    for (int l = lo; l < hi; l++) {
        atomicAdd(&vcnt[cell_at(g, l, x, y)], 1);
        g.dirty_commit[track_of(g, l, x, y, layer_first)] = 1;
    }
}

template <int G, int T>
__global__ void __launch_bounds__(128) pattern_route_kernel(GridDev g, TreeBatchDev b, int stamp) {
    extern __shared__ unsigned char smem_raw[];
    constexpr int kGroups = 128 / G;
    constexpr int kNodeTile = T;
    GroupSmem<T> &sm = reinterpret_cast<GroupSmem<T> *>(smem_raw)[threadIdx.x / G];
    __shared__ int layer_first[kL + 1];
    if (threadIdx.x == 0) {
        int f = 0;
        for (int l = 0; l < g.L; l++) { layer_first[l] = f; f += layer_dir(g, l) ? g.X : g.Y; }
        layer_first[g.L] = f;
    }
    __syncthreads();
    (void)kGroups;
    const int lane = threadIdx.x & 31;
    const int gl = lane & (G - 1);                 // lane within the group
    const int g0 = lane & ~(G - 1);                // first lane of the group
    const unsigned gmask = G == 32 ? 0xffffffffu : (0xffffu << g0);
    const int X = g.X, Y = g.Y, XY = X * Y;

    while (true) {
        int k = 0;
        if (gl == 0) k = atomicAdd(b.queue, 1);
        k = __shfl_sync(gmask, k, g0);
        if (k >= b.n) break;
        const int net = b.net_ids[b.order ? b.order[k] : k];
        const int nb = b.node_off[net];
        const int n = b.node_off[net + 1] - nb;
        const int *nodes = b.nodes + nb;
        const int *par = b.par + nb;
        double *dist;
        float *col;
        short *from;
        int *lr, *nx, *ny, *nl, *np;
        if (n <= kNodeTile) {
            dist = sm.dist; col = sm.col; from = sm.from; lr = sm.lr;
            nx = sm.nx; ny = sm.ny; nl = sm.nl; np = sm.np;
        } else {
            const int64_t so = b.scratch_off[net];
            if (so < 0 || so + n > b.scratch_nodes) {
                if (gl == 0) set_error(g.err, so < 0 ? ERR_STATE : ERR_CAPACITY);
                continue;
            }
            dist = b.scratch + so * kPatternScratchD;
            int *ib = reinterpret_cast<int *>(b.scratch + b.scratch_nodes * kPatternScratchD) + so * kPatternScratchI;
            col = reinterpret_cast<float *>(ib);
            from = reinterpret_cast<short *>(ib + (int64_t)n * kCol);
            lr = ib + (int64_t)n * (kCol + (kR + 1) / 2);
            nx = lr + n; ny = nx + n; nl = ny + n; np = nl + n;
        }
        // ---- 0. node positions and parents, decoded once
        for (int i = gl; i < n; i += G) {
            const int v = nodes[i];
            const int l = v / XY, r = v - l * XY, x = r / Y;
            nx[i] = x; ny[i] = r - x * Y; nl[i] = l; np[i] = par[i];
        }
        __syncwarp(gmask);
        // ---- 1a. via columns of all nodes, every load in flight at once, then the
        //          via-stack cost of every node and layer range (Lshape_route.hpp:22-32)
        for (int p = gl; p < n * kCol; p += G) {
            const int i = p / kCol;
            col[p] = g.vcost[cell_at(g, p - i * kCol, nx[i], ny[i])];
        }
        __syncwarp(gmask);
        for (int p = gl; p < n * kL; p += G) {
            const int i = p / kL, mn = p % kL;
            const int l = nl[i];
            const float *cc = col + i * kCol;
            double acc = 0;
            dist[i * kR + tri(mn, mn)] = (l < kL && l != mn) ? kInf : 0.0;
            for (int mx = mn + 1; mx < kL; mx++) {
                acc = acc + (double)cc[mx - 1];
                dist[i * kR + tri(mn, mx)] = (l < kL && (mn > l || mx < l)) ? kInf : acc;
            }
        }
        // ---- 2. bottom-up over tree edges (Lshape_route.hpp:33-97).  The
        //      geometry-only costs of edge i-1 are loaded into registers while
        //      edge i is computed and stored into the other half of sm.pf after it.
        constexpr int kPer = (kPF + G - 1) / G;
        double q[kPer];
        auto load_edge = [&](int i) {
            int x = 0, y = 0, px = 0, py = 0;
            bool use = false;
            if (i >= 1) {
                const int pi = np[i];
                if (pi >= 0 && pi < i) { use = true; x = nx[i]; y = ny[i]; px = nx[pi]; py = ny[pi]; }
            }
#pragma unroll
            for (int u = 0; u < kPer; u++) {
                const int j = gl + u * G;
                q[u] = (use && j < kPF) ? edge_value(g, x, y, px, py, j) : 0.0;
            }
        };
        auto store_edge = [&](int i) {
            double *slot = sm.pf + (i & 1) * kPF;
#pragma unroll
            for (int u = 0; u < kPer; u++)
                if (gl + u * G < kPF) slot[gl + u * G] = q[u];
        };
        if (n > 1) {
            load_edge(n - 1);
            store_edge(n - 1);
        }
        __syncwarp(gmask);
        bool bad = false;
        for (int i = n - 1; i >= 1; i--) {
            const int pi = np[i];
            if (pi < 0 || pi >= i) { bad = true; break; }
            load_edge(i - 1);
            const int x = nx[i], y = ny[i], px = nx[pi], py = ny[pi];
            const double *nd = dist + i * kR;
            double *pd = dist + pi * kR;
            short *prev = from + i * kR;
            const double *pe = sm.pf + (i & 1) * kPF;
            // (a) cheapest range containing each layer
            double mcc = kInf;
            int cf = 0;
            if (gl < kL) {
                for (int mn = 0; mn <= gl; mn++)
                    for (int mx = gl; mx < kL; mx++) {
                        const double c = nd[tri(mn, mx)];
                        if (c < mcc) { mcc = c; cf = mn * kL + mx; }
                    }
            }
            if (x == px || y == py) {
                if (gl < kL) {
                    double d = kInf;
                    int pp = 0;
                    const int dl = layer_dir(g, gl);
                    if (!((dl == 0 && y != py) || (dl == 1 && x != px))) {
                        d = mcc + pe[gl];
                        pp = cf * kL * kL + gl * kL + gl;
                    }
                    sm.diag[gl] = d;
                    sm.pdiag[gl] = pp;
                }
            } else {
                if (gl < kL) {
                    double cost = mcc;
                    cost += pe[gl];
                    sm.costc[gl] = cost;
                    sm.cf[gl] = cf;
                }
                __syncwarp(gmask);
                if (gl < kL) {
                    const int p = gl;
                    const double legp = pe[kL + p];
                    double best = kInf;
                    int bp = 0;
                    for (int c = (p & 1) ^ 1; c < kL; c += 2) {
                        const int lo = min(c, p), hi = max(c, p);
                        const double *vc = layer_dir(g, c) ? pe + 2 * kL : pe + 3 * kL;
                        double cost2 = 0;
                        for (int l = lo + 1; l < hi; l++) cost2 += vc[l];
                        cost2 += legp;
                        const double cand = sm.costc[c] + cost2;
                        if (cand < best) { best = cand; bp = sm.cf[c] * kL * kL + c * kL + p; }
                    }
                    sm.diag[p] = best;
                    sm.pdiag[p] = bp;
                }
            }
            __syncwarp(gmask);
            // (b) range minimum with the reference's <= rule, then accumulate into the parent
            if (gl < kL) {
                const int mn = gl;
                double row = sm.diag[mn];
                int rp = sm.pdiag[mn];
                prev[tri(mn, mn)] = rp;
                pd[tri(mn, mn)] += row;
                for (int mx = mn + 1; mx < kL; mx++) {
                    const double dg = sm.diag[mx];
                    if (!(row <= dg)) { row = dg; rp = sm.pdiag[mx]; }
                    prev[tri(mn, mx)] = rp;
                    pd[tri(mn, mx)] += row;
                }
            }
            store_edge(i - 1);
            __syncwarp(gmask);
        }
        if (bad) {
            if (gl == 0) set_error(g.err, ERR_STATE);
            __syncwarp(gmask);
            continue;
        }
        // ---- 3. root range: first minimum in (minl, maxl) order (Lshape_route.hpp:99-105)
        double bv = __longlong_as_double(0x7ff0000000000000LL);  // +infinity
        int bi = 1 << 30;
        for (int t = gl; t < kR; t += G) {
            const double c = dist[t];
            if (c < bv || (c == bv && t < bi)) { bv = c; bi = t; }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(gmask, bv, o, G);
            const int oi = __shfl_down_sync(gmask, bi, o, G);
            if (ov < bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        // ---- 4. backtrace, route emission and demand (Lshape_route.hpp:99-152).
        //      One lane walks the nodes in preorder and fixes each node's layer
        //      range from its parent's (shared memory only), stopping at the
        //      first node without a finite range; then every lane takes nodes:
        //      the segments of a node (its via stack, then the straight wire or
        //      the leg, corner via and leg of a bend) get their positions in the
        //      record from a prefix sum over nodes, in the reference's order, and
        //      the demand of each segment that fits the record is applied.
        __shared__ int s_stop[128 / G];
        if (gl == 0) {
            int rmn = 0, rmx = 0;
            for (int a = 0, t = 0; a < kL; a++)
                for (int c = a; c < kL; c++, t++)
                    if (t == bi) { rmn = a; rmx = c; }
            lr[0] = rmn * kL + rmx;
            int stop = n;
            for (int i = 0; i < n; i++) {
                if (i > 0) {
                    const int plr = lr[np[i]];
                    lr[i] = from[i * kR + tri(plr / kL, plr % kL)] / (kL * kL);
                }
                const int mn = lr[i] / kL, mx = lr[i] % kL;
                if (mn > mx || !(dist[i * kR + tri(mn, mx)] < kInf)) { stop = i; break; }
            }
            s_stop[threadIdx.x / G] = stop;
        }
        __syncwarp(gmask);
        const int stop = s_stop[threadIdx.x / G];
        int *r = b.routes + b.route_off[net];
        const int cap = b.route_cap[net];
        const int smax = cap >= 1 ? (cap - 1) / 2 : 0;  // segments that fit the record
        // segments of node i: emit(k, a, b, kind) for k = 0.. in record order;
        // kind 0: via stack at the node, 1: wire (l, xa, xb, ya, yb), 2: corner via
        auto node_segments = [&](int i, auto &&emit) {
            const int x = nx[i], y = ny[i];
            const int mn = lr[i] / kL, mx = lr[i] % kL;
            int k = 0;
            if (mn < mx) emit(k++, mn * XY + x * Y + y, mx * XY + x * Y + y, 0, mn, mx, x, y, 0);
            if (i == 0) return k;
            const int plr = lr[np[i]];
            const int code = from[i * kR + tri(plr / kL, plr % kL)];
            const int px = nx[np[i]], py = ny[np[i]];
            const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
            const int curl = code / kL % kL, parl = code % kL;
            const int vlo = min(curl, parl), vhi = max(curl, parl);
            if (px == x || py == y) {
                emit(k++, curl * XY + minx * Y + miny, curl * XY + maxx * Y + maxy, 1, curl, minx, maxx, miny, maxy);
            } else if (layer_dir(g, curl)) {
                emit(k++, curl * XY + x * Y + y, curl * XY + x * Y + py, 1, curl, x, x, miny, maxy);
                emit(k++, curl * XY + x * Y + py, parl * XY + x * Y + py, 2, vlo, vhi, x, py, 0);
                emit(k++, parl * XY + x * Y + py, parl * XY + px * Y + py, 1, parl, minx, maxx, py, py);
            } else {
                emit(k++, curl * XY + x * Y + y, curl * XY + px * Y + y, 1, curl, minx, maxx, y, y);
                emit(k++, curl * XY + px * Y + y, parl * XY + px * Y + y, 2, vlo, vhi, px, y, 0);
                emit(k++, parl * XY + px * Y + y, parl * XY + px * Y + py, 1, parl, px, px, miny, maxy);
            }
            return k;
        };
        auto no_emit = [](int, int, int, int, int, int, int, int, int) {};
        int carry = 0;  // segments of the nodes before this round
        long long nvias = 0;
        for (int i0 = 0; i0 < stop; i0 += G) {
            const int i = i0 + gl;
            const int cnt = i < stop ? node_segments(i, no_emit) : 0;
            int inc = cnt;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) {
                const int t = __shfl_up_sync(gmask, inc, o, G);
                if (gl >= o) inc += t;
            }
            const int first = carry + inc - cnt;  // global index of this node's first segment
            if (i < stop && first < smax) {
                node_segments(i, [&](int k, int a, int c, int kind, int p0, int p1, int p2, int p3, int p4) {
                    const int sidx = first + k;
                    if (sidx >= smax) return;
                    r[1 + 2 * sidx] = a;
                    r[2 + 2 * sidx] = c;
                    if (kind == 1) {
                        add_wire(g, layer_first, p0, p1, p2, p3, p4, stamp);
                    } else if (b.vcnt) {  // kinds 0 and 2: a via stack from layer p0 to p1 at (p2, p3)
                        count_vias(g, b.vcnt, layer_first, p0, p1, p2, p3);
                        nvias += p1 - p0;
                    }
                });
            }
            carry += __shfl_sync(gmask, inc, G - 1, G);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) nvias += __shfl_down_sync(gmask, nvias, o, G);
        if (gl == 0) {
            // the reference meets whichever comes first: a record overflow at a node
            // before `stop` ends the walk there; otherwise the state error at `stop`
            if (carry > smax) set_error(g.err, ERR_CAPACITY);
            else if (stop < n) set_error(g.err, ERR_STATE);
            r[0] = 1 + 2 * min(carry, smax);
            if (nvias) atomicAdd(&g.stats[1], (unsigned long long)nvias);
        }
        __syncwarp(gmask);
    }
}

template <int G, int T>
void launch_g(const GridDev &g, const TreeBatchDev &b, int stamp, cudaStream_t s) {
    constexpr int kThreads = 128;
    const size_t smem = sizeof(GroupSmem<T>) * (kThreads / G);
    const KernelShape ks = kernel_setup((const void *)pattern_route_kernel<G, T>, kThreads, smem);
    const int sms = ks.sms, per = ks.blocks_per_sm;
    const int groups_per_block = kThreads / G;
    int blocks = (b.n + groups_per_block - 1) / groups_per_block;
    if (blocks > sms * per) blocks = sms * per;
    if (blocks < 1) blocks = 1;
    pattern_route_kernel<G, T><<<blocks, kThreads, smem, s>>>(g, b, stamp);
}

}  // namespace

// Tile sizes (nodes kept on chip per group) compiled in: 6 (small nets), 16,
// 32 (32 lanes only) and 1 (every net in global scratch).
void launch_pattern_route(const GridDev &g, const TreeBatchDev &b, int stamp, cudaStream_t s) {
    if (b.n <= 0) return;
    const bool half = b.lanes_per_net == 16;
    switch (b.tile) {
        case 6: half ? launch_g<16, 6>(g, b, stamp, s) : launch_g<32, 6>(g, b, stamp, s); break;
        case 1: half ? launch_g<16, 1>(g, b, stamp, s) : launch_g<32, 1>(g, b, stamp, s); break;
        case 32: launch_g<32, 32>(g, b, stamp, s); break;
        default: half ? launch_g<16, 16>(g, b, stamp, s) : launch_g<32, 16>(g, b, stamp, s); break;
    }
}

}  // namespace igr
