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
#include <type_traits>

namespace igr {

namespace {

constexpr int kTrackThreads = 256;

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

// of_cost_scaled (graph.hpp:23-27, of_cost_scale = 1) in float: the
// reference's exponent arguments 0.5 * (d - c) and 1.5 * d are formed in
// double from float operands, where both products are exact, and rounded to
// float, which is the correctly rounded float product 0.5f * (d - c) or
// 1.5f * d; the comparison with 0.001 stays in double.
__device__ __forceinline__ float of_cost_f(bool has_cap, float c, float d) {
    if (has_cap) return __expf(0.5f * (d - c));
    return d > 0.f ? __expf(1.5f * d) : 0.f;
}

// Cost model and Sklansky prefix sums of one track of n cells whose capacity
// and demand are staged in s_cap / s_dem (and s_of1 has room for n floats);
// every thread of the block calls it and tallies n in g.stats[slot].  Cell i lives at thread i % T, row i / T.
//
// Each cell's overflow costs at demand d, d + 0.5 and d + 1 are evaluated once
// and left in shared memory (over its staged capacity and demand), so that
// cell i reads its left neighbour's instead of evaluating them again:
// vcost(i) needs the half-unit costs of cells i-1 and i, the wire cost of edge
// i-1 the unit cost of cell i-1 (graph.hpp:40-71).
template <int T, int MAXE>
__device__ __forceinline__ void refresh_track(const GridDev &g, const TrackInfo &ti, float *s_cap, float *s_dem,
                                              float *s_of1, int slot) {
    constexpr int W = T / 32;
    const int n = ti.len;
    const int E = (n + T - 1) / T;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double sc = g.short_cost[ti.l];
    const int *elen = ti.dir ? g.ylen : g.xlen;
    __shared__ double s_wt[W][MAXE];
    __shared__ double s_rt[MAXE];
    if (tid == 0) atomicAdd(&g.stats[slot], (unsigned long long)n);  // refreshed cells, for the roofline

#pragma unroll
    for (int r = 0; r < MAXE; r++) {
        const int i = tid + r * T;
        if (r < E && i < n) {
            const float c = s_cap[i], d = s_dem[i];
            const bool has_cap = (double)c > 0.001;
            const double dd = (double)d;
            s_cap[i] = of_cost_f(has_cap, c, d);
            s_dem[i] = of_cost_f(has_cap, c, (float)(dd + 0.5));
            s_of1[i] = of_cost_f(has_cap, c, (float)(dd + 1.0));
        }
    }
    __syncthreads();
    double x[MAXE];
#pragma unroll
    for (int r = 0; r < MAXE; r++) {
        x[r] = 0;
        const int i = tid + r * T;
        if (r < E && i < n) {
            const double of0 = (double)s_cap[i];
            const double bh = fmin(1e12, ((double)s_dem[i] - of0) * sc);
            float v;
            if (i == 0) {
                v = (float)fmin(1e12, ((double)s_of1[0] - of0) * sc);
            } else {
                const double ofp = (double)s_cap[i - 1];
                const double a1p = fmin(1e12, ((double)s_of1[i - 1] - ofp) * sc);
                if (i == n - 1) {
                    v = (float)a1p;
                } else {
                    const double bhp = fmin(1e12, ((double)s_dem[i - 1] - ofp) * sc);
                    v = (float)(bh + bhp);
                }
                // scan input: wire cost of edge i-1 (graph.hpp:44-46)
                float w = (float)a1p;
                w = (float)fma(g.unit_wire, (double)elen[i - 1], (double)w);
                x[r] = (double)w;
            }
            v = (float)((double)v + g.unit_via);
            g.vcost[ti.base + i] = v;
        }
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
    // ---- levels 5..log2(T)-1: warps
#pragma unroll
    for (int m = 0; (1 << m) < W; m++) {
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
    // ---- levels >= log2(T): rows
    if (E > 1) {
        if (tid == T - 1) {
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
        const int i = tid + r * T;
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

// Threads per track of the per-track kernels: five CTAs of 256 per SM (a
// CTA of 512 or 1024 threads per track shortens each track's chain but keeps
// fewer tracks in flight per SM, and the refresh is issue-bound: 17.2 and
// 28.2 ms against 11.5 ms per route of the 800k-net design).
#define IGR_TRACK_BOUNDS(T) __launch_bounds__(T, 5)

template <int T, int MAXE>
__global__ void IGR_TRACK_BOUNDS(T) cost_refresh_kernel(GridDev g, int only_dirty) {
    chain_begin();
    const int tr = blockIdx.x;
    if (only_dirty) {
        if (!g.dirty_cost[tr]) return;
    }
    const TrackInfo ti = decode_track(g, tr);
    extern __shared__ __align__(16) float s_track[];  // capacity, demand, unit-step cost: MAXE * T each
    float *s_cap = s_track, *s_dem = s_track + MAXE * T, *s_of1 = s_track + 2 * MAXE * T;
    stage_track(g.cap + ti.base, g.demand + ti.base, s_cap, s_dem, ti.len, threadIdx.x, T);
    __syncthreads();
    if (threadIdx.x == 0 && only_dirty) g.dirty_cost[tr] = 0;
    refresh_track<T, MAXE>(g, ti, s_cap, s_dem, s_of1, 2);
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
template <int T, int MAXE>
__global__ void IGR_TRACK_BOUNDS(T) commit_refresh_kernel(GridDev g, int *vcnt, int stamp, int refresh) {
    extern __shared__ __align__(16) float s_track[];  // capacity, demand, unit-step cost: MAXE * T each
    float *s_cap = s_track, *s_dem = s_track + MAXE * T, *s_of1 = s_track + 2 * MAXE * T;
    __shared__ int s_w[T / 32];
    __shared__ int s_carry;
    __shared__ long long s_wl[T / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tr = blockIdx.x;
    const bool commit = g.dirty_commit[tr] != 0;
    if (!commit && !(refresh && g.dirty_cost[tr])) return;
    const TrackInfo ti = decode_track(g, tr);
    const int n = ti.len;
    stage_track(refresh ? g.cap + ti.base : nullptr, g.demand + ti.base, s_cap, s_dem, n, tid, T);
    if (commit) {
        const int *elen = ti.dir ? g.ylen : g.xlen;
        if (tid == 0) s_carry = 0;
        __syncthreads();
        long long wl = 0;
        for (int r0 = 0; r0 < n; r0 += T) {
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
            if (tid == T - 1) s_carry = cnt;
            __syncthreads();
        }
        // vias, after every wire stamp of the track is in place
        for (int i = tid; i < n; i += T) {
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
        for (int i = tid; i < n; i += T) g.demand[ti.base + i] = s_dem[i];
        if (tid == 0) {
            long long t = 0;
            for (int w = 0; w < T / 32; w++) t += s_wl[w];
            if (t) atomicAdd(&g.stats[0], (unsigned long long)t);
            atomicAdd(&g.stats[3], (unsigned long long)n);  // committed cells, for the roofline
            g.dirty_commit[tr] = 0;
            g.dirty_cost[tr] = refresh ? 0 : 1;
        }
    } else {
        __syncthreads();
        if (tid == 0) g.dirty_cost[tr] = 0;
    }
    if (refresh) refresh_track<T, MAXE>(g, ti, s_cap, s_dem, s_of1, 4);
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

// dynamic shared memory of a track kernel: capacity, demand and unit-step
// cost of T * E cells
template <int T, int E>
constexpr size_t track_smem() { return (size_t)3 * T * E * sizeof(float); }

// One CTA per track: the hardware block scheduler hands the dirty tracks to
// the SMs as they free up, and a CTA that finds its track clean exits at once
// (a resident grid striding over the tracks balanced the uneven dirty tracks
// worse: 11.9 -> 15.8 ms per route of the 800k-net design; a resident grid
// over a list of the dirty tracks made by a one-CTA pass saved nothing).
template <int T, int E>
static void cost_refresh_e(const GridDev &g, int od, cudaStream_t s) {
    constexpr size_t smem = track_smem<T, E>();
    kernel_setup((const void *)cost_refresh_kernel<T, E>, T, smem);
    launch_chained(cost_refresh_kernel<T, E>, dim3(g.ntracks), dim3(T), smem, s, g, od);
}

template <int T, int E>
static void commit_refresh_e(const GridDev &g, int *vcnt, int stamp, int rf, cudaStream_t s) {
    constexpr size_t smem = track_smem<T, E>();
    kernel_setup((const void *)commit_refresh_kernel<T, E>, T, smem);
    commit_refresh_kernel<T, E><<<g.ntracks, T, smem, s>>>(g, vcnt, stamp, rf);
}

// Calls f(E) with E = the rows per thread of a 256-thread CTA for tracks of
// maxlen <= kMaxFusedTrackCells cells, exactly ceil(maxlen / 256): rows that
// hold no cell of any track would still be scanned.
template <int E, class F>
static void with_rows(int e, F &&f) {
    if constexpr (E * kTrackThreads >= kMaxFusedTrackCells) {
        f(std::integral_constant<int, E>());
    } else {
        if (e <= E) f(std::integral_constant<int, E>());
        else with_rows<E + 1>(e, f);
    }
}

void launch_cost_refresh(const GridDev &g, bool only_dirty, cudaStream_t s) {
    const int maxlen = g.X > g.Y ? g.X : g.Y;
    const int od = only_dirty ? 1 : 0;
    if (maxlen <= kMaxFusedTrackCells) {
        with_rows<1>((maxlen + kTrackThreads - 1) / kTrackThreads,
                     [&](auto ec) { cost_refresh_e<kTrackThreads, decltype(ec)::value>(g, od, s); });
    } else {
        const size_t smem = (size_t)kMaxTrackCells * 8;
        kernel_setup((const void *)cost_refresh_long_kernel, kLongThreads, smem);
        cost_refresh_long_kernel<<<g.ntracks, kLongThreads, smem, s>>>(g, od);
    }
}

void launch_commit_refresh(const GridDev &g, int *vcnt, int stamp, bool refresh, cudaStream_t s) {
    const int maxlen = g.X > g.Y ? g.X : g.Y;
    if (maxlen > kMaxFusedTrackCells) throw Error(ERR_STATE, "fused batch commit on tracks longer than 4096 cells");
    const int rf = refresh ? 1 : 0;
    with_rows<1>((maxlen + kTrackThreads - 1) / kTrackThreads,
                 [&](auto ec) { commit_refresh_e<kTrackThreads, decltype(ec)::value>(g, vcnt, stamp, rf, s); });
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
void launch_to_track_layout_i(const GridDev &g, const int *ref, int *trk, cudaStream_t s) {
    ref_to_track_kernel<int><<<grid_for(g.N), 256, 0, s>>>(g, ref, trk);
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
