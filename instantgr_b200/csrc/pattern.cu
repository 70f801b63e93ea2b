// Phase-1 pattern routing: layer-assignment DP over each net's Steiner tree
// with straight and L-shaped edges, then backtrace, route emission and demand
// difference-array updates.
//
// Restates Lshape_route_cuda (src/Lshape_route.hpp:9-153).  The reference runs
// one thread per net with 81-entry f64 tables per node in global memory (928
// bytes of stack per thread).  Here one warp owns a net: the 45 valid
// layer-range entries of every node live in shared memory (global scratch for
// nets with more than kNodeTile nodes), and the lanes of the warp work on the
// nine layers, the nine layer ranges and the 4-5 bend layers of one tree edge
// at a time.  All f64 sums are formed in the reference's order and every
// comparison keeps its strict/non-strict tie rule, so for the same cost map
// the chosen layers, routes and demand are bit-identical to the reference's.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kL = kRouteL;         // 9 routing layers
constexpr int kR = 45;              // layer ranges minl <= maxl
constexpr int kNodeTile = kPatternNodeTile;  // nodes kept on chip per warp
constexpr int kWarps = 4;           // warps per CTA

__host__ __device__ constexpr int tri(int a, int b) { return a * 9 - a * (a - 1) / 2 + (b - a); }

struct WarpSmem {
    double dist[kNodeTile * kR];
    int from[kNodeTile * kR];
    int lr[kNodeTile];
    double costc[kL], vA[kL], vB[kL], diag[kL];
    int cf[kL], pdiag[kL];
};

__device__ __forceinline__ double wire_cost(const GridDev &g, int l, int xa, int xb, int ya, int yb) {
    // presum[IDX(l, xmax, ymax)] - presum[IDX(l, xmin, ymin)]  (graph.hpp:19-21)
    return g.presum[cell_at(g, l, xb, yb)] - g.presum[cell_at(g, l, xa, ya)];
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

__global__ void __launch_bounds__(kWarps * 32) pattern_route_kernel(GridDev g, TreeBatchDev b, int stamp) {
    extern __shared__ unsigned char smem_raw[];
    WarpSmem &sm = reinterpret_cast<WarpSmem *>(smem_raw)[threadIdx.x >> 5];
    __shared__ int layer_first[kL + 1];
    if (threadIdx.x == 0) {
        int f = 0;
        for (int l = 0; l < g.L; l++) { layer_first[l] = f; f += layer_dir(g, l) ? g.X : g.Y; }
        layer_first[g.L] = f;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int X = g.X, Y = g.Y, XY = X * Y;

    for (int k = gw; k < b.n; k += nw) {
        const int net = b.net_ids[k];
        const int nb = b.node_off[net];
        const int n = b.node_off[net + 1] - nb;
        const int *nodes = b.nodes + nb;
        const int *par = b.par + nb;
        double *dist;
        int *from, *lr;
        if (n <= kNodeTile) {
            dist = sm.dist; from = sm.from; lr = sm.lr;
        } else {
            const int64_t so = b.scratch_off[net];
            if (so < 0) { set_error(g.err, ERR_STATE); continue; }
            if (so + n > b.scratch_nodes) { set_error(g.err, ERR_CAPACITY); continue; }
            dist = b.scratch + so * kR;
            from = reinterpret_cast<int *>(b.scratch + b.scratch_nodes * kR) + so * (kR + 1);
            lr = from + (int64_t)n * kR;
        }
        // ---- 1. via-stack cost of every node and layer range (Lshape_route.hpp:22-32)
        for (int p = lane; p < n * kL; p += 32) {
            const int i = p / kL, mn = p % kL;
            const int v = nodes[i];
            const int l = v / XY, x = v / Y % X, y = v % Y;
            double acc = 0;
            dist[i * kR + tri(mn, mn)] = (l < kL && l != mn) ? kInf : 0.0;
            for (int mx = mn + 1; mx < kL; mx++) {
                acc = acc + (double)g.vcost[cell_at(g, mx - 1, x, y)];
                dist[i * kR + tri(mn, mx)] = (l < kL && (mn > l || mx < l)) ? kInf : acc;
            }
        }
        __syncwarp();
        // ---- 2. bottom-up over tree edges (Lshape_route.hpp:33-97)
        for (int i = n - 1; i >= 1; i--) {
            const int pi = par[i];
            if (pi < 0 || pi >= i) { set_error(g.err, ERR_STATE); break; }
            const int v = nodes[i], pv = nodes[pi];
            const int x = v / Y % X, y = v % Y, px = pv / Y % X, py = pv % Y;
            const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
            const double *nd = dist + i * kR;
            double *pd = dist + pi * kR;
            int *prev = from + i * kR;
            // (a) cheapest range containing each layer
            double mcc = kInf;
            int cf = 0;
            if (lane < kL) {
                for (int mn = 0; mn <= lane; mn++)
                    for (int mx = lane; mx < kL; mx++) {
                        const double c = nd[tri(mn, mx)];
                        if (c < mcc) { mcc = c; cf = mn * kL + mx; }
                    }
            }
            const bool straight = (x == px || y == py);
            if (straight) {
                if (lane < kL) {
                    double d = kInf;
                    int pp = 0;
                    const int dl = layer_dir(g, lane);
                    if (!((dl == 0 && y != py) || (dl == 1 && x != px))) {
                        d = mcc + wire_cost(g, lane, minx, maxx, miny, maxy);
                        pp = cf * kL * kL + lane * kL + lane;
                    }
                    sm.diag[lane] = d;
                    sm.pdiag[lane] = pp;
                }
            } else {
                if (lane < kL) {
                    const int c = lane;
                    double cost = mcc;
                    if (layer_dir(g, c)) cost += wire_cost(g, c, x, x, miny, maxy);
                    else cost += wire_cost(g, c, minx, maxx, y, y);
                    sm.costc[c] = cost;
                    sm.cf[c] = cf;
                    sm.vA[lane] = (double)g.vcost[cell_at(g, lane, x, py)];
                } else if (lane < 2 * kL) {
                    sm.vB[lane - kL] = (double)g.vcost[cell_at(g, lane - kL, px, y)];
                }
                double legp = 0;
                if (lane < kL) {
                    if (layer_dir(g, lane)) legp = wire_cost(g, lane, px, px, miny, maxy);
                    else legp = wire_cost(g, lane, minx, maxx, py, py);
                }
                __syncwarp();
                if (lane < kL) {
                    const int p = lane;
                    double best = kInf;
                    int bp = 0;
                    for (int c = (p & 1) ^ 1; c < kL; c += 2) {
                        const int lo = min(c, p), hi = max(c, p);
                        const double *vc = layer_dir(g, c) ? sm.vA : sm.vB;
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
            __syncwarp();
            // (b) range minimum with the reference's <= rule, then accumulate into the parent
            if (lane < kL) {
                const int mn = lane;
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
            __syncwarp();
        }
        // ---- 3. root range: first minimum in (minl, maxl) order (Lshape_route.hpp:99-105)
        double bv = __longlong_as_double(0x7ff0000000000000LL);  // +infinity
        int bi = 1 << 30;
        for (int t = lane; t < kR; t += 32) {
            const double c = dist[t];
            if (c < bv || (c == bv && t < bi)) { bv = c; bi = t; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov < bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        // ---- 4. backtrace, route emission and demand (Lshape_route.hpp:99-152)
        if (lane == 0) {
            int *r = b.routes + b.route_off[net];
            const int cap = b.route_cap[net];
            int cnt = 1;
            bool ok = true;
            auto emit = [&](int a, int c) {
                if (cnt + 2 > cap) { ok = false; return; }
                r[cnt++] = a;
                r[cnt++] = c;
            };
            // root range as (minl, maxl)
            int rmn = 0, rmx = 0;
            for (int a = 0, t = 0; a < kL; a++)
                for (int c = a; c < kL; c++, t++)
                    if (t == bi) { rmn = a; rmx = c; }
            lr[0] = rmn * kL + rmx;
            for (int i = 0; i < n && ok; i++) {
                const int v = nodes[i];
                const int x = v / Y % X, y = v % Y;
                int code = 0;
                if (i > 0) {
                    const int plr = lr[par[i]];
                    code = from[i * kR + tri(plr / kL, plr % kL)];
                    lr[i] = code / (kL * kL);
                }
                const int mn = lr[i] / kL, mx = lr[i] % kL;
                if (mn > mx || !(dist[i * kR + tri(mn, mx)] < kInf)) { set_error(g.err, ERR_STATE); ok = false; break; }
                if (mn < mx) emit(mn * XY + x * Y + y, mx * XY + x * Y + y);
                if (i == 0) continue;
                const int pv = nodes[par[i]];
                const int px = pv / Y % X, py = pv % Y;
                const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
                const int curl = code / kL % kL, parl = code % kL;
                if (px == x || py == y) {
                    emit(curl * XY + minx * Y + miny, curl * XY + maxx * Y + maxy);
                    add_wire(g, layer_first, curl, minx, maxx, miny, maxy, stamp);
                } else if (layer_dir(g, curl)) {
                    emit(curl * XY + x * Y + y, curl * XY + x * Y + py);
                    add_wire(g, layer_first, curl, x, x, miny, maxy, stamp);
                    emit(curl * XY + x * Y + py, parl * XY + x * Y + py);
                    emit(parl * XY + x * Y + py, parl * XY + px * Y + py);
                    add_wire(g, layer_first, parl, minx, maxx, py, py, stamp);
                } else {
                    emit(curl * XY + x * Y + y, curl * XY + px * Y + y);
                    add_wire(g, layer_first, curl, minx, maxx, y, y, stamp);
                    emit(curl * XY + px * Y + y, parl * XY + px * Y + y);
                    emit(parl * XY + px * Y + y, parl * XY + px * Y + py);
                    add_wire(g, layer_first, parl, px, px, miny, maxy, stamp);
                }
            }
            if (!ok) set_error(g.err, ERR_CAPACITY);
            r[0] = cnt;
        }
        __syncwarp();
    }
}

}  // namespace

void launch_pattern_route(const GridDev &g, const TreeBatchDev &b, int stamp, cudaStream_t s) {
    if (b.n <= 0) return;
    const size_t smem = sizeof(WarpSmem) * kWarps;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(pattern_route_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    int blocks = (b.n + kWarps - 1) / kWarps;
    if (blocks > 148 * 8) blocks = 148 * 8;
    pattern_route_kernel<<<blocks, kWarps * 32, smem, s>>>(g, b, stamp);
}

}  // namespace igr
