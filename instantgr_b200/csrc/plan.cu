// Phase-1 routing plan built on the device from the colouring result.
//
// The colouring leaves a batch id per rank; InstantGR routes the batches in
// reverse order (Lshape_route.hpp:176) and, within a batch, in any order
// (the nets of a batch are independent).  The plan lists the routing-net ids
// batch by batch (routing order), each batch split into the size classes of
// the tree DP (large, medium, small) with the nets of a class by node count,
// largest first, so that the long nets of a launch start early.  It is a
// counting sort over (batch, class, node-count bucket) keys: histogram,
// exclusive scan, scatter.  The order within one key is arbitrary, which
// changes no result.
#include "kcommon.cuh"

#include <algorithm>

namespace igr {

namespace {

constexpr int kPlanBuckets = 64;  // node-count buckets per class (nets with more nodes share the first)
constexpr int kScanThreads = 1024;

__device__ __forceinline__ int plan_key(const PlanArgs &a, int k) {
    const int b = a.bat[k];
    const int id = a.perm ? a.perm[k] : k;
    const int m = a.node_off[id + 1] - a.node_off[id];
    const int c = a.classes == 1 ? 1 : (m > a.big ? 0 : (m > a.split ? 1 : 2));
    const int rb = a.nb - 1 - b;
    return (rb * 3 + c) * kPlanBuckets + (kPlanBuckets - 1 - min(m, kPlanBuckets - 1));
}

__global__ void plan_hist_kernel(PlanArgs a, int *hist, int *err) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x) {
        const int b = a.bat[k];
        if (b < 0 || b >= a.nb) {
            set_error(err, ERR_STATE);
            continue;
        }
        atomicAdd(hist + plan_key(a, k), 1);
    }
}

// Exclusive scan of hist[0..K) in place (one block), and the class offsets:
// offs[3 * rb + c] = first position of class c of routed batch rb, offs[3 * nb] = n.
__global__ void __launch_bounds__(kScanThreads) plan_scan_kernel(int K, int nb, int *hist, int *offs) {
    __shared__ int part[kScanThreads];
    const int t = threadIdx.x;
    const int chunk = (K + kScanThreads - 1) / kScanThreads;
    const int lo = min(K, t * chunk), hi = min(K, lo + chunk);
    int sum = 0;
    for (int i = lo; i < hi; i++) sum += hist[i];
    part[t] = sum;
    __syncthreads();
    for (int d = 1; d < kScanThreads; d <<= 1) {
        const int v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - sum;
    for (int i = lo; i < hi; i++) {
        const int c = hist[i];
        hist[i] = run;
        if (i % kPlanBuckets == 0) offs[i / kPlanBuckets] = run;
        run += c;
    }
    if (t == kScanThreads - 1) offs[3 * nb] = part[t];
}

__global__ void plan_scatter_kernel(PlanArgs a, int *cursor, int *ids) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x) {
        const int b = a.bat[k];
        if (b < 0 || b >= a.nb) continue;
        ids[atomicAdd(cursor + plan_key(a, k), 1)] = a.perm ? a.perm[k] : k;
    }
}

}  // namespace

int64_t plan_hist_size(int nb) { return (int64_t)nb * 3 * kPlanBuckets; }

void launch_plan(const PlanArgs &a, int *hist, int *ids, int *offs, int *err, cudaStream_t s) {
    if (a.n <= 0 || a.nb <= 0) return;
    const int K = (int)plan_hist_size(a.nb);
    cudaMemsetAsync(hist, 0, sizeof(int) * (size_t)K, s);
    const int blocks = std::min(1184, (a.n + 255) / 256);
    plan_hist_kernel<<<blocks, 256, 0, s>>>(a, hist, err);
    plan_scan_kernel<<<1, kScanThreads, 0, s>>>(K, a.nb, hist, offs);
    plan_scatter_kernel<<<blocks, 256, 0, s>>>(a, hist, ids);
}

}  // namespace igr
