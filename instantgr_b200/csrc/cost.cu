// Fused congestion-cost refresh: wire cost, via cost and the per-track prefix
// sums of wire cost, in one pass over each track.
//
// Replaces three full-grid kernels of InstantGR (update_wcost_cuda_ispd24,
// update_vcost_ispd24, compute_presum; src/graph.hpp:40-71, :101-104,
// :405-430).  One CTA of 256 threads owns one track: it stages the track's
// capacity and demand in shared memory with coalesced loads, evaluates the
// cost model for every cell, writes vcost (f32), and scans the wire costs in
// f64 into presum.  The wire cost array itself is never written: 20 bytes of
// DRAM traffic per cell (4+4 read, 4+8 written) instead of the reference's
// >= 44.
//
// The prefix sum keeps the exact association of the reference's in-place
// Sklansky scan (at level d, element i with bit d set adds element
// ((i >> d) << d) - 1), so presum is bit-identical to the reference's for the
// same demand.  Element i sits at thread i % 256, row i / 256: levels 0-4 are
// lane shuffles, levels 5-7 go through shared memory between warps, and levels
// >= 8 combine whole rows, whose running totals every thread tracks itself.
#include "kcommon.cuh"
#include "host.hpp"

#include <algorithm>
#include <cstdint>

namespace igr {

namespace {

constexpr int kThreads = 256;

// Cost model of cell i of a track staged in s_cap / s_dem: writes its via cost
// and returns the scan input, the wire cost of edge i-1 (0 for i = 0).
__device__ __forceinline__ double cell_costs(const GridDev &g, const TrackInfo &ti, const float *s_cap,
                                             const float *s_dem, int i, double sc, const int *elen) {
    const int n = ti.len;
    const float c = s_cap[i], d = s_dem[i];
    const double of0 = of_cost(c, d);
    const double bh = fmin(1e12, (of_cost(c, (float)((double)d + 0.5)) - of0) * sc);
    float v;
    double x = 0;
    if (i == 0) {
        v = (float)fmin(1e12, (of_cost(c, (float)((double)d + 1.0)) - of0) * sc);
    } else {
        const float cp = s_cap[i - 1], dp = s_dem[i - 1];
        const double ofp = of_cost(cp, dp);
        const double a1p = fmin(1e12, (of_cost(cp, (float)((double)dp + 1.0)) - ofp) * sc);
        if (i == n - 1) {
            v = (float)a1p;
        } else {
            const double bhp = fmin(1e12, (of_cost(cp, (float)((double)dp + 0.5)) - ofp) * sc);
            v = (float)(bh + bhp);
        }
        // scan input: wire cost of edge i-1 (graph.hpp:44-46)
        float w = (float)a1p;
        w = (float)fma(g.unit_wire, (double)elen[i - 1], (double)w);
        x = (double)w;
    }
    v = (float)((double)v + g.unit_via);
    g.vcost[ti.base + i] = v;
    return x;
}

// Cost model and Sklansky prefix sums of one track whose capacity and demand
// are staged in s_cap / s_dem; every thread of the block calls it.
template <int MAXE>
__device__ __forceinline__ void refresh_track(const GridDev &g, const TrackInfo &ti, const float *s_cap,
                                              const float *s_dem) {
    const int n = ti.len;
    const int E = (n + kThreads - 1) / kThreads;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double sc = g.short_cost[ti.l];
    const int *elen = ti.dir ? g.ylen : g.xlen;
    __shared__ double s_wt[kThreads / 32][MAXE];
    __shared__ double s_rt[MAXE];
    if (tid == 0) atomicAdd(&g.stats[2], (unsigned long long)n);  // refreshed cells, for the roofline

    double x[MAXE];
#pragma unroll
    for (int r = 0; r < MAXE; r++) {
        x[r] = 0;
        const int i = tid + r * kThreads;
        if (r < E && i < n) x[r] = cell_costs(g, ti, s_cap, s_dem, i, sc, elen);
    }
    // ---- Sklansky levels 0..4: lanes
#pragma unroll
    for (int m = 0; m < 5; m++) {
        const int src = ((lane >> m) << m) - 1;
        const bool take = (lane >> m) & 1;
#pragma unroll
        for (int r = 0; r < MAXE; r++) {
            double o = __shfl_sync(0xffffffffu, x[r], src & 31);
            if (take) x[r] += o;
        }
    }
    // ---- levels 5..7: warps
#pragma unroll
    for (int m = 0; m < 3; m++) {
        if (lane == 31) {
#pragma unroll
            for (int r = 0; r < MAXE; r++) s_wt[warp][r] = x[r];
        }
        __syncthreads();
        if ((warp >> m) & 1) {
            const int sw = ((warp >> m) << m) - 1;
#pragma unroll
            for (int r = 0; r < MAXE; r++) x[r] += s_wt[sw][r];
        }
        __syncthreads();
    }
    // ---- levels >= 8: rows
    if (E > 1) {
        if (tid == kThreads - 1) {
#pragma unroll
            for (int r = 0; r < MAXE; r++) s_rt[r] = x[r];
        }
        __syncthreads();
        double rt[MAXE];
#pragma unroll
        for (int r = 0; r < MAXE; r++) rt[r] = s_rt[r];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            if ((1 << m) >= MAXE) break;
#pragma unroll
            for (int r = 0; r < MAXE; r++) {
                if ((r >> m) & 1) {
                    const int sr = ((r >> m) << m) - 1;
                    x[r] += rt[sr];
                    rt[r] += rt[sr];
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < MAXE; r++) {
        const int i = tid + r * kThreads;
        if (r < E && i < n) g.presum[ti.base + i] = x[r];
    }
}

// Copies n floats of a track's capacity (when `a` is non-null) and demand into
// shared memory in one loop, so that the loads of both arrays are in flight
// together: 16 bytes per load where the track starts on a 16-byte boundary
// (every track of a grid whose X*Y and track lengths are multiples of 4), else
// one float per load.
__device__ __forceinline__ void stage_track(const float *a, const float *b, float *da, float *db, int n, int tid,
                                            int nthreads) {
    if ((reinterpret_cast<uintptr_t>(b) & 15) == 0) {
        const int n4 = n >> 2;
        const float4 *a4 = reinterpret_cast<const float4 *>(a), *b4 = reinterpret_cast<const float4 *>(b);
        float4 *da4 = reinterpret_cast<float4 *>(da), *db4 = reinterpret_cast<float4 *>(db);
        for (int i = tid; i < n4; i += nthreads) {
            const float4 vb = b4[i];
            if (a) da4[i] = a4[i];
            db4[i] = vb;
        }
        for (int i = (n4 << 2) + tid; i < n; i += nthreads) {
            if (a) da[i] = a[i];
            db[i] = b[i];
        }
    } else {
        for (int i = tid; i < n; i += nthreads) {
            if (a) da[i] = a[i];
            db[i] = b[i];
        }
    }
}

template <int MAXE>
__global__ void __launch_bounds__(kThreads, 5) cost_refresh_kernel(GridDev g, int only_dirty) {
    const int tr = blockIdx.x;
    if (only_dirty) {
        if (!g.dirty_cost[tr]) return;
    }
    const TrackInfo ti = decode_track(g, tr);
    __shared__ __align__(16) float s_cap[MAXE * kThreads];
    __shared__ __align__(16) float s_dem[MAXE * kThreads];
    stage_track(g.cap + ti.base, g.demand + ti.base, s_cap, s_dem, ti.len, threadIdx.x, kThreads);
    __syncthreads();
    if (threadIdx.x == 0 && only_dirty) g.dirty_cost[tr] = 0;
    refresh_track<MAXE>(g, ti, s_cap, s_dem);
}

// Tracks of more than 4096 cells (up to the reference's 15,360, main.cpp:28):
// a CTA of kLongThreads per track, the costs evaluated into registers, then
// the reference's in-place Sklansky scan level by level in shared memory
// (graph.hpp:421-428; at level d an element reads an element whose bit d is
// clear, which that level never writes).  The f64 scan array reuses the
// shared memory of the staged capacity and demand.
constexpr int kLongThreads = 1024;
constexpr int kLongMaxE = kMaxTrackCells / kLongThreads;  // 15

__global__ void __launch_bounds__(kLongThreads) cost_refresh_long_kernel(GridDev g, int only_dirty) {
    extern __shared__ __align__(16) unsigned char long_smem[];
    float *s_cap = reinterpret_cast<float *>(long_smem);
    float *s_dem = s_cap + kMaxTrackCells;
    double *s_x = reinterpret_cast<double *>(long_smem);  // after the costs: 8 bytes per cell
    const int tid = threadIdx.x;
    const int tr = blockIdx.x;
    if (only_dirty && !g.dirty_cost[tr]) return;
    {
        const TrackInfo ti = decode_track(g, tr);
        const int n = ti.len;
        stage_track(g.cap + ti.base, g.demand + ti.base, s_cap, s_dem, n, tid, kLongThreads);
        __syncthreads();
        if (tid == 0) {
            if (only_dirty) g.dirty_cost[tr] = 0;
            atomicAdd(&g.stats[2], (unsigned long long)n);
        }
        const double sc = g.short_cost[ti.l];
        const int *elen = ti.dir ? g.ylen : g.xlen;
        double x[kLongMaxE];
#pragma unroll
        for (int r = 0; r < kLongMaxE; r++) {
            const int i = tid + r * kLongThreads;
            x[r] = i < n ? cell_costs(g, ti, s_cap, s_dem, i, sc, elen) : 0.0;
        }
        __syncthreads();  // every read of the staged capacity and demand is done
#pragma unroll
        for (int r = 0; r < kLongMaxE; r++) {
            const int i = tid + r * kLongThreads;
            if (i < n) s_x[i] = x[r];
        }
        __syncthreads();
        for (int d = 0; (1 << d) < n; d++) {
            for (int i = tid; i < n; i += kLongThreads)
                if ((i >> d) & 1) s_x[i] += s_x[((i >> d) << d) - 1];
            __syncthreads();
        }
        for (int i = tid; i < n; i += kLongThreads) g.presum[ti.base + i] = s_x[i];
    }
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Batch commit and cost refresh of one track in one pass (phase 1): the wire
// difference array is scanned into demand and stamps (compute_presum_general
// + commit_all_edge, graph.hpp:74-137), the via crossings the tree DP counted
// per cell are added where this batch's wires left no stamp
// (commit_via_demand, graph.hpp:496-543: half a unit on each track edge
// beside the cell, a full unit at the track ends), and the costs and prefix
// sums are rebuilt from the demand still in shared memory.  Tracks with no
// pending commit and clean costs are skipped.  With refresh = 0 the costs are
// only marked dirty.
template <int MAXE>
__global__ void __launch_bounds__(kThreads, 5) commit_refresh_kernel(GridDev g, int *vcnt, int stamp, int refresh) {
    __shared__ __align__(16) float s_cap[MAXE * kThreads];
    __shared__ __align__(16) float s_dem[MAXE * kThreads];
    __shared__ int s_w[kThreads / 32];
    __shared__ int s_carry;
    __shared__ long long s_wl[kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tr = blockIdx.x;
    const bool commit = g.dirty_commit[tr] != 0;
    if (!commit && !(refresh && g.dirty_cost[tr])) return;
    const TrackInfo ti = decode_track(g, tr);
    const int n = ti.len;
    stage_track(refresh ? g.cap + ti.base : nullptr, g.demand + ti.base, s_cap, s_dem, n, tid, kThreads);
    if (commit) {
        const int *elen = ti.dir ? g.ylen : g.xlen;
        if (tid == 0) s_carry = 0;
        __syncthreads();
        long long wl = 0;
        for (int r0 = 0; r0 < n; r0 += kThreads) {
            const int i = r0 + tid;
            int v = 0;
            if (i < n) {
                v = g.pre[ti.base + i];
                if (v != 0) g.pre[ti.base + i] = 0;
            }
            const int inc = warp_incl_scan(v, lane);
            if (lane == 31) s_w[warp] = inc;
            __syncthreads();
            int wpre = 0;
            for (int w = 0; w < warp; w++) wpre += s_w[w];
            const int cnt = s_carry + wpre + inc;  // inclusive prefix at i
            if (i < n - 1 && cnt > 0) {
                s_dem[i] += (float)cnt;
                g.stamp[ti.base + i] = stamp;
                wl += (long long)cnt * elen[i];
            }
            __syncthreads();
            if (tid == kThreads - 1) s_carry = cnt;
            __syncthreads();
        }
        // vias, after every wire stamp of the track is in place
        for (int i = tid; i < n; i += kThreads) {
            const int c = vcnt[ti.base + i];
            if (c == 0) continue;
            vcnt[ti.base + i] = 0;
            if (g.stamp[ti.base + i] >= stamp) continue;
            if (i == 0) atomicAdd(&s_dem[0], (float)c);
            else if (i == n - 1) atomicAdd(&s_dem[n - 2], (float)c);
            else {
                atomicAdd(&s_dem[i - 1], 0.5f * (float)c);
                atomicAdd(&s_dem[i], 0.5f * (float)c);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wl += __shfl_down_sync(0xffffffffu, wl, o);
        if (lane == 0) s_wl[warp] = wl;
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) g.demand[ti.base + i] = s_dem[i];
        if (tid == 0) {
            long long t = 0;
            for (int w = 0; w < kThreads / 32; w++) t += s_wl[w];
            if (t) atomicAdd(&g.stats[0], (unsigned long long)t);
            atomicAdd(&g.stats[3], (unsigned long long)n);  // committed cells, for the roofline
            g.dirty_commit[tr] = 0;
            g.dirty_cost[tr] = refresh ? 0 : 1;
        }
    } else {
        __syncthreads();
        if (tid == 0) g.dirty_cost[tr] = 0;
    }
    if (refresh) refresh_track<MAXE>(g, ti, s_cap, s_dem);
}

template <typename T>
__global__ void ref_to_track_kernel(GridDev g, const T *ref, T *trk) {
    const int64_t n = g.N;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int l = (int)(k / ((int64_t)g.X * g.Y));
        int rem = (int)(k - (int64_t)l * g.X * g.Y);
        int x = rem / g.Y, y = rem % g.Y;
        trk[cell_at(g, l, x, y)] = ref[k];
    }
}

template <typename T>
__global__ void track_to_ref_kernel(GridDev g, const T *trk, T *ref) {
    const int64_t n = g.N;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int l = (int)(k / ((int64_t)g.X * g.Y));
        int rem = (int)(k - (int64_t)l * g.X * g.Y);
        int x = rem / g.Y, y = rem % g.Y;
        ref[k] = trk[cell_at(g, l, x, y)];
    }
}

}  // namespace

// One CTA per track: the hardware block scheduler hands the dirty tracks to
// the SMs as they free up (a resident grid striding over the tracks balanced
// the uneven dirty tracks worse: 11.9 -> 15.8 ms per step on the 800k-net
// design), and a CTA that finds its track clean exits at once.
template <int E>
static void cost_refresh_e(const GridDev &g, int od, cudaStream_t s) {
    cost_refresh_kernel<E><<<g.ntracks, kThreads, 0, s>>>(g, od);
}

void launch_cost_refresh(const GridDev &g, bool only_dirty, cudaStream_t s) {
    const int maxlen = g.X > g.Y ? g.X : g.Y;
    const int e = (maxlen + kThreads - 1) / kThreads;
    const int od = only_dirty ? 1 : 0;
    if (e <= 1) cost_refresh_e<1>(g, od, s);
    else if (e <= 2) cost_refresh_e<2>(g, od, s);
    else if (e <= 4) cost_refresh_e<4>(g, od, s);
    else if (e <= 8) cost_refresh_e<8>(g, od, s);
    else if (e <= 16) cost_refresh_e<16>(g, od, s);  // tracks of <= 4096 cells
    else {
        const size_t smem = (size_t)kMaxTrackCells * 8;
        kernel_setup((const void *)cost_refresh_long_kernel, kLongThreads, smem);
        cost_refresh_long_kernel<<<g.ntracks, kLongThreads, smem, s>>>(g, od);
    }
}

template <int E>
static void commit_refresh_e(const GridDev &g, int *vcnt, int stamp, int rf, cudaStream_t s) {
    commit_refresh_kernel<E><<<g.ntracks, kThreads, 0, s>>>(g, vcnt, stamp, rf);
}

void launch_commit_refresh(const GridDev &g, int *vcnt, int stamp, bool refresh, cudaStream_t s) {
    const int maxlen = g.X > g.Y ? g.X : g.Y;
    if (maxlen > kMaxFusedTrackCells) throw Error(ERR_STATE, "fused batch commit on tracks longer than 4096 cells");
    const int e = (maxlen + kThreads - 1) / kThreads;
    const int rf = refresh ? 1 : 0;
    if (e <= 1) commit_refresh_e<1>(g, vcnt, stamp, rf, s);
    else if (e <= 2) commit_refresh_e<2>(g, vcnt, stamp, rf, s);
    else if (e <= 4) commit_refresh_e<4>(g, vcnt, stamp, rf, s);
    else if (e <= 8) commit_refresh_e<8>(g, vcnt, stamp, rf, s);
    else commit_refresh_e<16>(g, vcnt, stamp, rf, s);  // longer tracks commit with the split launches
}

static int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

void launch_to_track_layout(const GridDev &g, const float *ref, float *trk, cudaStream_t s) {
    ref_to_track_kernel<float><<<grid_for(g.N), 256, 0, s>>>(g, ref, trk);
}
void launch_to_track_layout_d(const GridDev &g, const double *ref, double *trk, cudaStream_t s) {
    ref_to_track_kernel<double><<<grid_for(g.N), 256, 0, s>>>(g, ref, trk);
}
void launch_from_track_layout_i(const GridDev &g, const int *trk, int *ref, cudaStream_t s) {
    track_to_ref_kernel<int><<<grid_for(g.N), 256, 0, s>>>(g, trk, ref);
}
void launch_from_track_layout_f(const GridDev &g, const float *trk, float *ref, cudaStream_t s) {
    track_to_ref_kernel<float><<<grid_for(g.N), 256, 0, s>>>(g, trk, ref);
}
void launch_from_track_layout_d(const GridDev &g, const double *trk, double *ref, cudaStream_t s) {
    track_to_ref_kernel<double><<<grid_for(g.N), 256, 0, s>>>(g, trk, ref);
}

std::string cuda_error_string(cudaError_t e) { return cudaGetErrorString(e); }

}  // namespace igr
