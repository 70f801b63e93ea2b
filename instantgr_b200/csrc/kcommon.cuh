// Shared device helpers: grid layout, track decoding and the congestion cost
// model.  The cost arithmetic mirrors InstantGR's expression by expression
// (src/graph.hpp:19-71): float demand/capacity, double intermediate terms, the
// __expf intrinsic, and the same float roundings, so that the cost map of
// this project matches the reference's bit for bit for the same demand.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "device.hpp"

namespace igr {

constexpr double kInf = 1e22;     // the reference's INF (src/database_cuda.hpp:54)
constexpr int kRouteL = 9;        // routing layers handled by the DP kernels

__device__ __forceinline__ int layer_dir(const GridDev &g, int l) { return (l & 1) ^ g.DIR; }

// Programmatic dependent launch, first statement of the kernels of a reroute
// batch: the next kernel of the stream may be scheduled from now on, and this
// one waits until every kernel before it has finished and its writes are
// visible.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void chain_begin() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch with programmatic stream serialization: the kernel's CTAs may be
// scheduled while the previous kernel of the stream finishes (it hides the
// launch gaps between the short kernels of a reroute batch: 228.3 -> 226.6 ms
// per route of the 800k-net design, identical results); the kernel must start
// with chain_begin().
template <typename... KArgs, typename... Args>
inline void launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                           Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// offset of cell (l, x, y) in the track-contiguous layout
__device__ __forceinline__ int64_t cell_at(const GridDev &g, int l, int x, int y) {
    int64_t b = (int64_t)l * g.X * g.Y;
    return layer_dir(g, l) ? b + (int64_t)x * g.Y + y : b + (int64_t)y * g.X + x;
}

// track of cell (l, x, y): global track id
__device__ __forceinline__ int track_of(const GridDev &g, int l, int x, int y, const int *layer_first) {
    return layer_first[l] + (layer_dir(g, l) ? x : y);
}

struct TrackInfo {
    int l, t, len, dir;
    int64_t base;
};

__device__ __forceinline__ TrackInfo decode_track(const GridDev &g, int tr) {
    TrackInfo ti;
    int l = 0, first = 0;
    while (true) {
        int cnt = layer_dir(g, l) ? g.X : g.Y;
        if (tr < first + cnt || l == g.L - 1) { ti.t = tr - first; break; }
        first += cnt;
        l++;
    }
    ti.l = l;
    ti.dir = layer_dir(g, l);
    ti.len = ti.dir ? g.Y : g.X;
    ti.base = (int64_t)l * g.X * g.Y + (int64_t)ti.t * ti.len;
    return ti;
}

// of_cost_scaled (graph.hpp:23-27) with of_cost_scale = 1
__device__ __forceinline__ double of_cost(float capacity, float demand) {
    const double scale = 1.0;
    if (capacity > 0.001) {
        double t = 0.5 * (demand - capacity);
        double u = scale * 0.5 * (demand - capacity);
        return __expf((float)fmin(t, u));
    }
    if (demand > 0) {
        double t = 1.5 * demand;
        double u = scale * 1.5 * demand;
        return __expf((float)fmin(t, u));
    }
    return 0;
}

// incremental_of_cost (graph.hpp:34-38) with incre_base = 0
__device__ __forceinline__ double incr_cost(float c, float d, double inc, double short_cost) {
    float d1 = (float)((double)d + inc + 0.0);
    float d0 = (float)((double)d + 0.0);
    return fmin(1e12, (of_cost(c, d1) - of_cost(c, d0)) * short_cost);
}

__device__ __forceinline__ void set_error(int *err, int code) {
    if (err) atomicCAS(err, 0, code);
}

}  // namespace igr
