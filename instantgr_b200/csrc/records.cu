// Dense copy of the live route records, for the copy to the host.
//
// Route records are laid out with room for their largest possible size, and
// every rip-up pass appends a new record for each rerouted net, so only a
// small part of the record buffer is live once a run ends (on the 10M-net
// design about a tenth of 25 GB).  Before the records go to the host they are
// packed: the length of each net's record (its first entry), an exclusive scan
// into new offsets, and a copy, one warp per net.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kScanThreads = 1024;

// length of each record: its count, at least 1 (the count itself) and never
// past the end of the record buffer
__global__ void record_len_kernel(const int *routes, const int64_t *route_off, int n, int64_t end, int64_t *off) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t o = route_off[k];
    const int64_t len = o < end ? routes[o] : 1;
    off[k + 1] = len < 1 ? 1 : (len > end - o ? end - o : len);
}

// exclusive scan of a[1..n] into a[0..n] in one block (64-bit)
__global__ void __launch_bounds__(kScanThreads) record_scan_kernel(int64_t *a, int n) {
    __shared__ int64_t part[kScanThreads];
    const int t = threadIdx.x;
    const int chunk = (n + kScanThreads - 1) / kScanThreads;
    const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
    int64_t sum = 0;
    for (int i = lo; i < hi; i++) sum += a[i + 1];
    part[t] = sum;
    __syncthreads();
    for (int d = 1; d < kScanThreads; d <<= 1) {
        const int64_t v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int64_t run = part[t] - sum;
    for (int i = lo; i < hi; i++) {
        run += a[i + 1];
        a[i + 1] = run;
    }
    if (t == 0) a[0] = 0;
}

__global__ void take_i64_kernel(int n, const int *idx, const long long *src, long long *dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[idx[k]];
}

// new record slots of the rerouted nets: slot[k] = {id, offset, capacity}
__global__ void record_slots_kernel(int n, const int64_t *slot, int64_t *route_off, int *route_cap) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t id = slot[3 * k];
    route_off[id] = slot[3 * k + 1];
    route_cap[id] = (int)slot[3 * k + 2];
}

__global__ void record_copy_kernel(const int *routes, const int64_t *route_off, int n, const int64_t *off,
                                   int *dense) {
    const int lane = threadIdx.x & 31;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += (gridDim.x * blockDim.x) >> 5) {
        const int *r = routes + route_off[k];
        int *o = dense + off[k];
        const int len = (int)(off[k + 1] - off[k]);
        for (int i = lane; i < len; i += 32) o[i] = i ? r[i] : len;
    }
}

}  // namespace

void launch_record_offsets(const int *routes, const int64_t *route_off, int n, int64_t end, int64_t *off,
                           cudaStream_t s) {
    if (n > 0) record_len_kernel<<<(n + 255) / 256, 256, 0, s>>>(routes, route_off, n, end, off);
    record_scan_kernel<<<1, kScanThreads, 0, s>>>(off, n);
}

void launch_take_i64(int n, const int *idx, const long long *src, long long *dst, cudaStream_t s) {
    if (n > 0) take_i64_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, idx, src, dst);
}

void launch_record_slots(int n, const int64_t *slot, int64_t *route_off, int *route_cap, cudaStream_t s) {
    if (n > 0) record_slots_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, slot, route_off, route_cap);
}

void launch_record_copy(const int *routes, const int64_t *route_off, int n, const int64_t *off, int *dense,
                        cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (n + 7) / 8;
    if (blocks > 148 * 32) blocks = 148 * 32;
    record_copy_kernel<<<blocks, 256, 0, s>>>(routes, route_off, n, off, dense);
}

}  // namespace igr
