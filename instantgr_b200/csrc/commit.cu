// Demand commit: wires through the per-track difference array, vias and
// rip-up through exact float atomics.
//
//  * wire_commit: replaces compute_presum_general + commit_all_edge + the
//    cudaMemset of pre_demand (src/graph.hpp:74-99, :118-137).  One CTA per
//    track scans the integer difference array, adds the covered count to the
//    demand of every edge it spans, stamps those edges, accumulates the
//    wirelength and clears the array, in one pass; tracks without entries
//    are skipped through a per-track flag instead of sweeping the whole grid.
//  * via_commit: commit_via_demand (src/graph.hpp:496-543): each via span adds
//    half a unit of demand to the two track edges beside it (a full unit at
//    the track ends) on every layer it crosses whose cell this batch's wires
//    did not stamp.  One warp per net, lanes over route pairs.
//  * wire_ripup: commit_wire_demand with K = -1 (src/graph.hpp:468-495).
// Demand values are multiples of 0.5 far below 2^24, so the float atomics are
// exact and the result does not depend on their order.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__global__ void __launch_bounds__(kThreads) wire_commit_kernel(GridDev g, int stamp, int only_dirty) {
    chain_begin();
    const int tr = blockIdx.x;
    if (only_dirty && !g.dirty_commit[tr]) return;
    const TrackInfo ti = decode_track(g, tr);
    const int n = ti.len;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int *elen = ti.dir ? g.ylen : g.xlen;
    __shared__ int s_w[kThreads / 32];
    __shared__ int s_carry;
    __shared__ int s_any;
    if (tid == 0) { s_carry = 0; s_any = 0; }
    __syncthreads();
    long long wl = 0;
    int any = 0;
    for (int r0 = 0; r0 < n; r0 += kThreads) {
        const int i = r0 + tid;
        int v = 0;
        if (i < n) {
            v = g.pre[ti.base + i];
            if (v != 0) g.pre[ti.base + i] = 0;
        }
        int inc = warp_incl_scan(v, lane);
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        int wpre = 0;
        for (int w = 0; w < warp; w++) wpre += s_w[w];
        const int carry = s_carry;
        const int cnt = carry + wpre + inc;  // inclusive prefix at i
        if (i < n - 1 && cnt > 0) {
            const int64_t o = ti.base + i;
            g.demand[o] += (float)cnt;
            g.stamp[o] = stamp;
            wl += (long long)cnt * elen[i];
            any = 1;
        }
        __syncthreads();
        if (tid == kThreads - 1) s_carry = cnt;
        __syncthreads();
    }
    // block reduce of the wirelength
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wl += __shfl_down_sync(0xffffffffu, wl, o);
    __shared__ long long s_wl[kThreads / 32];
    if (lane == 0) s_wl[warp] = wl;
    if (any) s_any = 1;
    __syncthreads();
    if (tid == 0) {
        long long t = 0;
        for (int w = 0; w < kThreads / 32; w++) t += s_wl[w];
        if (t) atomicAdd(&g.stats[0], (unsigned long long)t);
        if (s_any) g.dirty_cost[tr] = 1;
        if (only_dirty) g.dirty_commit[tr] = 0;
    }
}

__device__ __forceinline__ void add_via_edge(const GridDev &g, int l, int x, int y, float v) {
    atomicAdd(&g.demand[cell_at(g, l, x, y)], v);
}

__device__ __forceinline__ void mark_cost_dirty(const GridDev &g, int l, int x, int y) {
    int first = 0;
    for (int k = 0; k < l; k++) first += layer_dir(g, k) ? g.X : g.Y;
    int tr = first + (layer_dir(g, l) ? x : y);
    if (!g.dirty_cost[tr]) g.dirty_cost[tr] = 1;
}

__global__ void via_commit_kernel(GridDev g, ViaBatchDev b, int stamp, int K) {
    chain_begin();
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int XY = g.X * g.Y;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < b.n; k += warps) {
        const int net = b.net_ids[k];
        const int *r = b.routes + b.route_off[net];
        const int cnt = r[0];
        long long vias = 0;
        for (int j = 1 + 2 * lane; j < cnt; j += 64) {
            const int a = r[j], c = r[j + 1];
            const int la = a / XY, lc = c / XY;
            if (la == lc) continue;
            const int x = a / g.Y % g.X, y = a % g.Y;
            const int mn = la < lc ? la : lc, mx = la < lc ? lc : la;
            vias += mx - mn;
            for (int l = mn; l < mx; l++) {
                if (g.stamp[cell_at(g, l, x, y)] >= stamp) continue;
                if (layer_dir(g, l)) {
                    if (y == 0) add_via_edge(g, l, x, y, (float)K);
                    else if (y == g.Y - 1) add_via_edge(g, l, x, y - 1, (float)K);
                    else { add_via_edge(g, l, x, y - 1, (float)(0.5 * K)); add_via_edge(g, l, x, y, (float)(0.5 * K)); }
                } else {
                    if (x == 0) add_via_edge(g, l, x, y, (float)K);
                    else if (x == g.X - 1) add_via_edge(g, l, x - 1, y, (float)K);
                    else { add_via_edge(g, l, x - 1, y, (float)(0.5 * K)); add_via_edge(g, l, x, y, (float)(0.5 * K)); }
                }
                mark_cost_dirty(g, l, x, y);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vias += __shfl_down_sync(0xffffffffu, vias, o);
        if (lane == 0 && vias) atomicAdd(&g.stats[1], (unsigned long long)(vias * K));
    }
}

__global__ void wire_ripup_kernel(GridDev g, ViaBatchDev b, int stamp, int K) {
    chain_begin();
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int XY = g.X * g.Y;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < b.n; k += warps) {
        const int net = b.net_ids[k];
        const int *r = b.routes + b.route_off[net];
        const int cnt = r[0];
        long long wl = 0;
        for (int j = 1 + 2 * lane; j < cnt; j += 64) {
            const int a = r[j], c = r[j + 1];
            const int l = a / XY;
            if (l != c / XY) continue;
            const int x0 = a / g.Y % g.X, y0 = a % g.Y, x1 = c / g.Y % g.X, y1 = c % g.Y;
            const int xa = x0 < x1 ? x0 : x1, xb = x0 < x1 ? x1 : x0;
            const int ya = y0 < y1 ? y0 : y1, yb = y0 < y1 ? y1 : y0;
            for (int x = xa; x < xb; x++) {
                atomicAdd(&g.demand[cell_at(g, l, x, y0)], (float)K);
                wl += g.xlen[x];
                g.stamp[cell_at(g, l, x, y0)] = stamp;
            }
            for (int y = ya; y < yb; y++) {
                atomicAdd(&g.demand[cell_at(g, l, x0, y)], (float)K);
                wl += g.ylen[y];
                g.stamp[cell_at(g, l, x0, y)] = stamp;
            }
            g.stamp[cell_at(g, l, x0, y0)] = stamp;
            g.stamp[cell_at(g, l, x0, y1)] = stamp;
            g.stamp[cell_at(g, l, x1, y0)] = stamp;
            g.stamp[cell_at(g, l, x1, y1)] = stamp;
            if (xa != xb || ya != yb) mark_cost_dirty(g, l, x0, y0);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wl += __shfl_down_sync(0xffffffffu, wl, o);
        if (lane == 0 && wl) atomicAdd(&g.stats[0], (unsigned long long)(wl * K));
    }
}

int warps_grid(int n) {
    int blocks = (n + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    return blocks < 1 ? 1 : blocks;
}

}  // namespace

void launch_wire_commit(const GridDev &g, int stamp, bool only_dirty, cudaStream_t s) {
    launch_chained(wire_commit_kernel, dim3(g.ntracks), dim3(kThreads), 0, s, g, stamp, only_dirty ? 1 : 0);
}

void launch_via_commit(const GridDev &g, const ViaBatchDev &b, int stamp, int K, cudaStream_t s) {
    if (b.n <= 0) return;
    launch_chained(via_commit_kernel, dim3(warps_grid(b.n)), dim3(256), 0, s, g, b, stamp, K);
}

void launch_wire_ripup(const GridDev &g, const ViaBatchDev &b, int stamp, int K, cudaStream_t s) {
    if (b.n <= 0) return;
    launch_chained(wire_ripup_kernel, dim3(warps_grid(b.n)), dim3(256), 0, s, g, b, stamp, K);
}

}  // namespace igr
