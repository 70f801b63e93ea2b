// Phase-2 DAG routing: per-edge mid-edge layer changes, the level-by-level
// DAG DP, the backtrace with route emission and demand, and a deterministic
// compaction of the emitted routes.
//
// Restates, with the reference's arithmetic and tie rules:
//   precompute_cost_edge                  src/Lshape_route_detour.hpp:123-195
//   Lshape_route_node_layer_change_cuda   src/Lshape_route_detour.hpp:281-406
//   get_routing_tree_layer_change_cuda    src/Lshape_route_detour.hpp:520-694
//   cost/id packing for atomicMin         src/Lshape_route_detour.hpp:83-112
// The reference launches two kernels per DAG level with a host synchronisation
// after each (2 x depth launches per batch).  Here one persistent cooperative
// kernel walks all levels of a batch, bottom-up then top-down, separated by a
// grid barrier that gives up after two seconds (ERR_TIMEOUT) rather than
// waiting forever.  Emitted segments are staged per DAG node and compacted in
// node order, so route records do not depend on atomic ordering (the
// reference appends them with atomicAdd).
#include "gridsync.cuh"

namespace igr {

namespace {

constexpr int kML = 10;                      // MAX_LAYER of the reference
constexpr unsigned long long kInitPacked = 7208259049189261824ULL;  // init_cost_with_road

__device__ __forceinline__ int32_t f2o(float f) {
    int32_t i = __float_as_int(f);
    return (i >= 0) ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int32_t i) { return __int_as_float((i >= 0) ? i : i ^ 0x7FFFFFFF); }
__device__ __forceinline__ unsigned long long pack(float cost, int id) {
    return ((unsigned long long)f2o(cost) << 32) | (unsigned int)id;
}
__device__ __forceinline__ void unpack(unsigned long long p, double *cost, int *id) {
    *cost = (double)o2f((int32_t)(p >> 32));
    *id = (int)(p & 0xFFFFFFFFull);
}

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

__global__ void dag_init_kernel(DagBatchDev b) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = tid; i < (int64_t)b.n_nodes * kML; i += nth) b.costs[i] = kInf;
    for (int64_t i = tid; i < (int64_t)b.n_slots * kML; i += nth) { b.packed[i] = kInitPacked; b.best_path[i] = 0; }
    for (int64_t i = tid; i < b.n_nodes; i += nth) { b.layer_out[i] = -1; b.stage_cnt[i] = 0; }
}

// precompute_cost_edge: one thread per (edge, from layer)
__global__ void dag_edge_cost_kernel(GridDev g, DagBatchDev b) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t e = idx / 9;
    if (e >= b.n_edges) return;
    const int f = (int)(idx % 9);
    const int to_node = b.par[e], from_node = b.edge_child[e];
    const int Y = g.Y, X = g.X;
    const int tox = b.nodes[to_node] / Y % X, toy = b.nodes[to_node] % Y;
    const int fx = b.nodes[from_node] / Y % X, fy = b.nodes[from_node] % Y;
    double *ce = b.cost_edges + e * 81 + f * 9;
    int *bc = b.best_change + e * 81 + f * 9;
    if ((layer_dir(g, f) == 0 && fy != toy) || (layer_dir(g, f) == 1 && fx != tox)) {
        for (int t = 0; t < 9; t++) ce[t] = kInf;
        return;
    }
    const int dist = abs(tox - fx) + abs(toy - fy);
    if (dist == 0) return;
    const int dd = dist / min(dist, 20);
    const bool vert = (fx == tox);
    const int s0 = vert ? min(fy, toy) : min(fx, tox);
    const int s1 = vert ? max(fy, toy) : max(fx, tox);
    for (int t = 0; t < 9; t++) {
        if ((t % 2) != (f % 2)) continue;
        double best = kInf;
        int pos = -1;
        for (int sp = s0 + dd; sp < s1; sp += dd) {
            const int sx = vert ? fx : sp, sy = vert ? sp : fy;
            double via = 0;
            for (int ll = min(f, t); ll < max(f, t); ll++) via += g.vcost[cell_at(g, ll, sx, sy)];
            double c = via;
            if (vert)
                c += (wire_cost(g, f, fx, fx, min(fy, sy), max(fy, sy)) + wire_cost(g, t, tox, tox, min(toy, sy), max(toy, sy)));
            else
                c += (wire_cost(g, f, min(fx, sx), max(fx, sx), fy, fy) + wire_cost(g, t, min(tox, sx), max(tox, sx), toy, toy));
            if (c < best) { best = c; pos = sp; }
        }
        ce[t] = best;
        bc[t] = pos;
    }
}

// Lshape_route_node_layer_change_cuda for one node
__device__ void dp_node(const GridDev &g, const DagBatchDev &b, int node) {
    const int X = g.X, Y = g.Y, XY = X * Y;
    const int pb = b.par_off[node], pn = b.par_off[node + 1] - pb;
    const int v = b.nodes[node];
    const int fixed_low = 1 + v / XY;
    const int x = v / Y % X, y = v % Y;
    const int fixed_high = fixed_low == 10 ? 0 : fixed_low;
    const int cb = b.child_off[node], cn = b.child_off[node + 1] - cb;
    unsigned long long *best = b.best_path + (int64_t)cb * kML;
    const unsigned long long *pk = b.packed + (int64_t)cb * kML;
    double *cost = b.costs + (int64_t)node * kML;
    double minc[kML];
    unsigned long long bp[kML];
    for (int c = 0; c < kML; c++) bp[c] = 0;
    for (int low = 1; low <= fixed_low; low++) {
        for (int c = 0; c < cn; c++) minc[c] = kInf;
        double via = 0;
        for (int layer = low; layer < g.L + 1; layer++) {
            if (layer > low) via += g.vcost[cell_at(g, layer - 2, x, y)];
            for (int c = 0; c < cn; c++) {
                double cc;
                int id;
                unpack(pk[c * kML + layer], &cc, &id);
                if (cc < minc[c]) { minc[c] = cc; bp[c] = (unsigned long long)id * kML + layer; }
            }
            if (layer >= fixed_high) {
                double t = via;
                for (int c = 0; c < cn; c++) t += minc[c];
                if (t < kInf && t < cost[layer]) {
                    cost[layer] = t;
                    for (int c = 0; c < cn; c++) best[c * kML + layer] = bp[c];
                }
            }
        }
        for (int layer = g.L + 1 - 2; layer >= low; layer--) {
            if (cost[layer + 1] < cost[layer]) {
                cost[layer] = cost[layer + 1];
                for (int c = 0; c < cn; c++) best[c * kML + layer] = best[c * kML + layer + 1];
            }
        }
    }
    for (int pi = 0; pi < pn; pi++) {
        const int e = pb + pi;
        const int parent = b.par[e];
        const int slot = b.child_slot[e];
        unsigned long long *ppk = b.packed + (int64_t)b.child_off[parent] * kML + slot * kML;
        const int pv = b.nodes[parent];
        const int px = pv / Y % X, py = pv % Y;
        const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
        unsigned long long cache[kML];
        for (int t = 1; t < kML; t++) cache[t] = ppk[t];
        for (int layer = 1; layer < kML; layer++) {
            const int dl = (layer & 1) ^ g.DIR;  // direction test of the reference, on 1-based layers
            if (dl == 1 && y != py) continue;
            if (dl == 0 && x != px) continue;
            const double base = cost[layer];
            for (int t = 1 + (1 - layer % 2); t < kML; t += 2) {
                double c2;
                int choice = 82;
                if (t == layer) {
                    c2 = base + wire_cost(g, layer - 1, minx, maxx, miny, maxy);
                } else if (abs(x - px) + abs(y - py) > 4) {
                    const int seq = (layer - 1) * 9 + (t - 1);
                    const double ce = b.cost_edges[(int64_t)e * 81 + seq];
                    if (ce < kInf) { c2 = base + ce; choice = seq; }
                    else continue;
                } else {
                    continue;
                }
                const unsigned long long nv = pack((float)c2, node * 100 + choice);
                if (nv < cache[t]) cache[t] = nv;
            }
        }
        for (int t = 1; t < kML; t++) atomicMin(ppk + t, cache[t]);
    }
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

__global__ void dag_levels_kernel(GridDev g, DagBatchDev b, unsigned *bar, int stamp) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    unsigned epoch = 0;
    for (int d = b.depth - 1; d >= 0; d--) {
        for (int s = b.level_off[d] + tid; s < b.level_off[d + 1]; s += nth) dp_node(g, b, b.level_nodes[s]);
        if (!grid_sync(bar, g.err, epoch)) return;
    }
    for (int d = 0; d < b.depth; d++) {
        for (int s = b.level_off[d] + tid; s < b.level_off[d + 1]; s += nth) trace_node(g, b, b.level_nodes[s], stamp);
        if (!grid_sync(bar, g.err, epoch)) return;
    }
}

// one-level launches, used when a cooperative launch is not available
__global__ void dag_dp_level_kernel(GridDev g, DagBatchDev b, int d) {
    const int s = b.level_off[d] + blockIdx.x * blockDim.x + threadIdx.x;
    if (s < b.level_off[d + 1]) dp_node(g, b, b.level_nodes[s]);
}
__global__ void dag_trace_level_kernel(GridDev g, DagBatchDev b, int d, int stamp) {
    const int s = b.level_off[d] + blockIdx.x * blockDim.x + threadIdx.x;
    if (s < b.level_off[d + 1]) trace_node(g, b, b.level_nodes[s], stamp);
}

// route records in DAG node order: one warp per net
__global__ void dag_compact_kernel(GridDev g, DagBatchDev b) {
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < b.n_nets; k += warps) {
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
}

}  // namespace

int launch_dag_route(const GridDev &g, const DagBatchDev &b, int stamp, unsigned *bar_words, bool cooperative,
                     cudaStream_t s) {
    if (b.n_nodes <= 0) return 0;
    int launches = 0;
    {
        int64_t work = (int64_t)b.n_slots * kML;
        if ((int64_t)b.n_nodes * kML > work) work = (int64_t)b.n_nodes * kML;
        int blocks = (int)((work + 255) / 256);
        if (blocks > 148 * 16) blocks = 148 * 16;
        dag_init_kernel<<<blocks < 1 ? 1 : blocks, 256, 0, s>>>(b);
        launches++;
    }
    if (b.n_edges > 0) {
        const int64_t th = (int64_t)b.n_edges * 9;
        dag_edge_cost_kernel<<<(int)((th + 255) / 256), 256, 0, s>>>(g, b);
        launches++;
    }
    if (cooperative) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dag_levels_kernel, 256, 0);
        int blocks = sms * (per < 2 ? per : 2);
        const int need = (int)((b.max_level + 255) / 256);
        if (need < blocks) blocks = need < 1 ? 1 : need;
        cudaMemsetAsync(bar_words, 0, 2 * sizeof(unsigned), s);
        unsigned *bar = bar_words;
        GridDev gg = g;
        DagBatchDev bb = b;
        void *args[] = {&gg, &bb, &bar, &stamp};
        cudaError_t e = cudaLaunchCooperativeKernel((const void *)dag_levels_kernel, dim3(blocks), dim3(256), args, 0, s);
        if (e != cudaSuccess) return -1;
        launches++;
    } else {
        for (int d = b.depth - 1; d >= 0; d--) {
            const int w = b.h_level_off[d + 1] - b.h_level_off[d];
            dag_dp_level_kernel<<<(w + 255) / 256, 256, 0, s>>>(g, b, d);
            launches++;
        }
        for (int d = 0; d < b.depth; d++) {
            const int w = b.h_level_off[d + 1] - b.h_level_off[d];
            dag_trace_level_kernel<<<(w + 255) / 256, 256, 0, s>>>(g, b, d, stamp);
            launches++;
        }
    }
    {
        int blocks = (b.n_nets + 7) / 8;
        if (blocks > 148 * 16) blocks = 148 * 16;
        dag_compact_kernel<<<blocks < 1 ? 1 : blocks, 256, 0, s>>>(g, b);
        launches++;
    }
    return launches;
}

}  // namespace igr
