// Rip-up selection, congestion view and overflow score.
//
//  * mark_overflow: mark_overflow_edges + compute_presum_general +
//    mark_overflow_nets (src/graph.hpp:432-466, :588-601).  One CTA per track
//    flags edges with cap + threshold <= demand and writes their exclusive
//    prefix count; then one warp per net counts flagged edges under its wires
//    and flags the net when the count exceeds `min_edges` (10 in the
//    reference).  The reference stops counting at the first prefix that
//    exceeds the limit; the total is compared here, which flags the same nets
//    because every segment adds a non-negative count.
//  * congestion view: extract_congestionView{,_xsum,_ysum}
//    (src/graph.hpp:545-584), the per-(x, y) maximum over layers of the
//    overflow (demand - cap)^+ followed by exclusive prefix sums along x and
//    along y.  The maximum is taken per cell by one thread (the reference
//    races on it), and the arrays start from zero (the reference never clears
//    them).  Overflows are multiples of 0.5, so the float sums are exact in
//    any order.
//  * overflow cost: add_all_overflow_cost (src/graph.hpp:148-157), reduced in a
//    fixed order (per track, then over tracks) instead of with f64 atomics.
//  * flag list: the indices of the flagged nets in increasing order, so that
//    only the list goes to the host: per-block counts, their exclusive scan,
//    then each block writes its indices from its offset.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int warp_incl_scan_i(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__global__ void __launch_bounds__(kThreads) overflow_edges_kernel(GridDev g, int threshold, int *of_sum) {
    const TrackInfo ti = decode_track(g, blockIdx.x);
    const int n = ti.len, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ int s_w[kThreads / 32];
    __shared__ int s_carry;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int r0 = 0; r0 < n; r0 += kThreads) {
        const int i = r0 + tid;
        int v = 0;
        if (i < n - 1) {
            const int64_t o = ti.base + i;
            v = (g.cap[o] + (float)threshold <= g.demand[o]) ? 1 : 0;
        }
        int inc = warp_incl_scan_i(v, lane);
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        int wpre = 0;
        for (int w = 0; w < warp; w++) wpre += s_w[w];
        const int carry = s_carry;
        if (i < n) of_sum[ti.base + i] = carry + wpre + inc - v;  // exclusive
        __syncthreads();
        if (tid == kThreads - 1) s_carry = carry + wpre + inc;
        __syncthreads();
    }
}

__global__ void overflow_nets_kernel(GridDev g, const int *of_sum, ViaBatchDev b, int min_edges, uint8_t *is_of) {
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int XY = g.X * g.Y;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < b.n; k += warps) {
        const int net = b.net_ids[k];
        const int *r = b.routes + b.route_off[net];
        const int cnt = r[0];
        int c = 0;
        for (int j = 1 + 2 * lane; j < cnt; j += 64) {
            const int a = r[j], e = r[j + 1];
            const int l = a / XY, x0 = a / g.Y % g.X, y0 = a % g.Y, x1 = e / g.Y % g.X, y1 = e % g.Y;
            if (x0 != x1) c += of_sum[cell_at(g, l, max(x0, x1), y0)] - of_sum[cell_at(g, l, min(x0, x1), y0)];
            if (y0 != y1) c += of_sum[cell_at(g, l, x0, max(y0, y1))] - of_sum[cell_at(g, l, x0, min(y0, y1))];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) is_of[k] = c > min_edges ? 1 : 0;
    }
}

__global__ void congestion_max_kernel(GridDev g, float *xsum, float *ysum) {
    const int XY = g.X * g.Y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < XY; k += gridDim.x * blockDim.x) {
        const int x = k / g.Y, y = k % g.Y;
        float m = 0.f;
        for (int l = 0; l < g.L; l++) {
            const int64_t o = cell_at(g, l, x, y);
            const double res = (double)(g.cap[o] - g.demand[o]);
            if (res < 0) m = fmaxf(m, (float)(-res));
        }
        xsum[k] = m;
        ysum[k] = m;
    }
}

// exclusive prefix along one axis: line `ln` of `cnt` elements with stride `st`
__global__ void __launch_bounds__(kThreads) view_scan_kernel(float *a, int cnt, int64_t st, int64_t lstride) {
    float *p = a + blockIdx.x * lstride;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ float s_w[kThreads / 32];
    __shared__ float s_carry;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int r0 = 0; r0 < cnt; r0 += kThreads) {
        const int i = r0 + tid;
        float v = (i < cnt - 1) ? p[i * st] : 0.f;  // element i feeds prefix i+1
        float inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            float t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        float wpre = 0;
        for (int w = 0; w < warp; w++) wpre += s_w[w];
        const float carry = s_carry;
        __syncthreads();
        if (i < cnt) p[i * st] = carry + wpre + inc - v;
        if (tid == kThreads - 1) s_carry = carry + wpre + inc;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) overflow_cost_kernel(GridDev g, double *partial) {
    const TrackInfo ti = decode_track(g, blockIdx.x);
    const int n = ti.len, tid = threadIdx.x;
    const double sc = g.short_cost[ti.l];
    double acc = 0;
    for (int i = tid; i < n - 1; i += kThreads) {
        const int64_t o = ti.base + i;
        acc += sc * of_cost(g.cap[o], g.demand[o]);
    }
    __shared__ double s[kThreads];
    s[tid] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (tid < w) s[tid] += s[tid + w];
        __syncthreads();
    }
    if (tid == 0) partial[blockIdx.x] = s[0];
}

__global__ void sum_partials_kernel(const double *partial, int n, double *out) {
    __shared__ double s[kThreads];
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += kThreads) acc += partial[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

int warps_grid(int n) {
    int blocks = (n + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    return blocks < 1 ? 1 : blocks;
}

}  // namespace

namespace {

constexpr int kFlagItems = 8;  // flags per thread of the list kernels
constexpr int kFlagBlock = kThreads * kFlagItems;

// flags [t * 8, t * 8 + 8) of the block's range, counted per thread
__device__ __forceinline__ int flag_count8(const uint8_t *flags, int n, int base, int t) {
    int c = 0;
#pragma unroll
    for (int j = 0; j < kFlagItems; j++) {
        const int i = base + t * kFlagItems + j;
        c += i < n && flags[i];
    }
    return c;
}

// exclusive scan of v over the block's threads; *total gets the block's sum
__device__ __forceinline__ int block_excl_scan(int v, int *total) {
    __shared__ int s_w[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int inc = warp_incl_scan_i(v, lane);
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
        const int x = lane < kThreads / 32 ? s_w[lane] : 0;
        const int xi = warp_incl_scan_i(x, lane);
        if (lane < kThreads / 32) s_w[lane] = xi - x;
        if (lane == kThreads / 32 - 1) *total = xi;
    }
    __syncthreads();
    return s_w[w] + inc - v;
}

__global__ void __launch_bounds__(kThreads) flag_count_kernel(const uint8_t *flags, int n, int *block_cnt) {
    __shared__ int s_total;
    const int c = flag_count8(flags, n, blockIdx.x * kFlagBlock, threadIdx.x);
    block_excl_scan(c, &s_total);
    if (threadIdx.x == 0) block_cnt[blockIdx.x] = s_total;
}

// exclusive scan of block_cnt[0..nb) in place (one block); the total to *count
__global__ void __launch_bounds__(kThreads) flag_offsets_kernel(int *block_cnt, int nb, int *count) {
    __shared__ int s_total;
    const int per = (nb + kThreads - 1) / kThreads;
    const int lo = min(nb, (int)threadIdx.x * per), hi = min(nb, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; i++) sum += block_cnt[i];
    int run = block_excl_scan(sum, &s_total);
    for (int i = lo; i < hi; i++) {
        const int c = block_cnt[i];
        block_cnt[i] = run;
        run += c;
    }
    if (threadIdx.x == 0) *count = s_total;
}

__global__ void __launch_bounds__(kThreads) flag_write_kernel(const uint8_t *flags, int n, const int *block_off,
                                                              int *list) {
    __shared__ int s_total;
    const int base = blockIdx.x * kFlagBlock, t = threadIdx.x;
    int at = block_off[blockIdx.x] + block_excl_scan(flag_count8(flags, n, base, t), &s_total);
#pragma unroll
    for (int j = 0; j < kFlagItems; j++) {
        const int i = base + t * kFlagItems + j;
        if (i < n && flags[i]) list[at++] = i;
    }
}

}  // namespace

int flag_list_blocks(int n) { return (n + kFlagBlock - 1) / kFlagBlock; }

void launch_flag_list(const uint8_t *flags, int n, int *list, int *count, int *block_cnt, cudaStream_t s) {
    const int nb = flag_list_blocks(n);
    if (nb == 0) {
        cudaMemsetAsync(count, 0, sizeof(int), s);
        return;
    }
    flag_count_kernel<<<nb, kThreads, 0, s>>>(flags, n, block_cnt);
    flag_offsets_kernel<<<1, kThreads, 0, s>>>(block_cnt, nb, count);
    flag_write_kernel<<<nb, kThreads, 0, s>>>(flags, n, block_cnt, list);
}

void launch_mark_overflow(const GridDev &g, int threshold, int *of_sum, const ViaBatchDev &nets, int min_edges,
                          uint8_t *is_of, cudaStream_t s) {
    overflow_edges_kernel<<<g.ntracks, kThreads, 0, s>>>(g, threshold, of_sum);
    if (nets.n > 0) overflow_nets_kernel<<<warps_grid(nets.n), 256, 0, s>>>(g, of_sum, nets, min_edges, is_of);
}

void launch_congestion_view(const GridDev &g, float *xsum, float *ysum, cudaStream_t s) {
    const int XY = g.X * g.Y;
    int blocks = (XY + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    congestion_max_kernel<<<blocks, 256, 0, s>>>(g, xsum, ysum);
    // xsum: for each y, along x (stride Y); ysum: for each x, along y (stride 1)
    view_scan_kernel<<<g.Y, kThreads, 0, s>>>(xsum, g.X, g.Y, 1);
    view_scan_kernel<<<g.X, kThreads, 0, s>>>(ysum, g.Y, 1, g.Y);
}

void launch_overflow_cost(const GridDev &g, double *out, cudaStream_t s) {
    // `out` must hold ntracks + 1 doubles: per-track partials, then the total
    overflow_cost_kernel<<<g.ntracks, kThreads, 0, s>>>(g, out + 1);
    sum_partials_kernel<<<1, kThreads, 0, s>>>(out + 1, g.ntracks, out);
}

}  // namespace igr
