// Phase-1 tree DP for callers that cannot allocate device memory.
//
// The tree DP keeps the layer tables of nets with more than kPatternNodeTile
// nodes in global scratch, and every launch needs a work counter, a per-net
// scratch offset and a net-id list.  igr_pattern_route gets these from
// cudaMalloc'd staging buffers.  Some callers cannot let a library allocate:
// a host that hands the GPU's memory to its own pool allocator and forbids
// other allocations, a real-time loop where a cudaMalloc (which can
// synchronise the device) would stall the other streams, or a process that
// runs close to the memory limit and must know its footprint up front.  For
// them this file holds the scratch in one fixed array in the library's own
// device image, so a call allocates nothing.
//
// Layout of the array (byte offsets, each part 256-byte aligned):
//   [0, 256)           StaticHeader (status, work counter, scratch node count)
//   [256, ...)         net ids 0..n-1 (int32)
//   [..., ...)         scratch offset per net (int64, -1 for nets kept on chip)
//   [..., capacity)    layer tables of the nets kept in scratch (doubles)
// The header is cleared at the start of every call; the rest is rewritten by
// every call before it is read.
#include "kcommon.cuh"
#include "router.hpp"

#include <mutex>
#include <string>

namespace igr {

namespace {

// One array per device that loads the library, held until the process exits.
static __device__ __align__(256) unsigned char g_pattern_scratch[kStaticScratchBytes];

struct StaticHeader {
    int status;      // OR of Bad* flags below
    int queue;       // work counter of the DP launch
    int bad_net;     // a net that failed validation
    int pad;
    long long big_nodes;  // nodes of the nets kept in scratch
};

enum : int { kBadOffsets = 1, kBadNode = 2, kBadParent = 4, kBadRecord = 8 };

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

constexpr int kPrepThreads = 1024;

// Net ids, node_off validation and the scratch offsets of nets larger than
// `tile` (an exclusive scan over the nets in one block).
__global__ void __launch_bounds__(kPrepThreads)
static_prep_kernel(int n, const int *node_off, long long total_nodes, int tile, StaticHeader *h, int *ids,
                   long long *so) {
    __shared__ long long part[kPrepThreads];
    const int t = threadIdx.x;
    const int chunk = (n + kPrepThreads - 1) / kPrepThreads;
    const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
    long long sum = 0;
    bool ok = true;
    for (int k = lo; k < hi; k++) {
        const int cnt = node_off[k + 1] - node_off[k];
        if (cnt < 1) ok = false;
        if (cnt > tile) sum += cnt;
    }
    if (t == 0 && (node_off[0] != 0 || node_off[n] != total_nodes)) ok = false;
    if (!ok) {
        atomicOr(&h->status, kBadOffsets);
        atomicExch(&h->bad_net, lo);
    }
    part[t] = sum;
    __syncthreads();
    for (int d = 1; d < kPrepThreads; d <<= 1) {
        const long long v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = part[t] - sum;
    for (int k = lo; k < hi; k++) {
        const int cnt = node_off[k + 1] - node_off[k];
        ids[k] = k;
        if (cnt > tile) {
            so[k] = run;
            run += cnt;
        } else {
            so[k] = -1;
        }
    }
    if (t == kPrepThreads - 1) h->big_nodes = part[t];
}

// Node positions, preorder parents and route-record bounds, one thread per net.
// Runs only over offsets that static_prep_kernel accepted.
__global__ void static_check_kernel(int n, const int *node_off, const int *nodes, const int *par,
                                    const int64_t *route_off, const int *route_cap, long long routes_len,
                                    long long cells, StaticHeader *h) {
    if (h->status & kBadOffsets) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int bad = 0;
        const long long ro = route_off[k];
        const int rc = route_cap[k];
        if (ro < 0 || rc < 1 || ro + rc > routes_len) bad |= kBadRecord;
        const int a = node_off[k], b = node_off[k + 1];
        for (int i = a; i < b; i++) {
            const int loc = i - a;
            if (nodes[i] < 0 || nodes[i] >= cells) bad |= kBadNode;
            if (loc == 0 ? par[i] != -1 : (par[i] < 0 || par[i] >= loc)) bad |= kBadParent;
        }
        if (bad) {
            atomicOr(&h->status, bad);
            atomicExch(&h->bad_net, k);
        }
    }
}

std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kStaticMaxDevices] = {};

// Device address of g_pattern_scratch on the current device, looked up once
// per device.  In host code the symbol names a host-side shadow, never the
// device memory, so it is not handed to a kernel itself.
unsigned char *static_scratch_ptr() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kStaticMaxDevices) throw Error(ERR_INVALID, "device ordinal beyond the static scratch table");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_pattern_scratch);
        if (e != cudaSuccess || !p)
            throw Error(ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
    }
    return g_scratch_ptr[dev];
}

}  // namespace

void pattern_route_static(const GridDev &g, int n, const int *node_off, int64_t total_nodes, const int *nodes,
                          const int *par, const int64_t *route_off, const int *route_cap, int *routes,
                          int64_t routes_len, int stamp, cudaStream_t s) {
    if (n < 0 || total_nodes < 0 || routes_len < 0) throw Error(ERR_INVALID, "negative size");
    if (n > kStaticMaxNets)
        throw Error(ERR_CAPACITY, "batch of " + std::to_string(n) + " nets exceeds the static-scratch limit of " +
                                      std::to_string(kStaticMaxNets) + " nets per call");
    if (n == 0) return;
    if (!node_off || !nodes || !par || !route_off || !route_cap || !routes) throw Error(ERR_INVALID, "null pointer");
    unsigned char *base = static_scratch_ptr();
    const size_t off_ids = 256;
    const size_t off_so = align256(off_ids + sizeof(int) * (size_t)n);
    const size_t off_tab = align256(off_so + sizeof(long long) * (size_t)n);
    auto *h = reinterpret_cast<StaticHeader *>(base);
    auto *ids = reinterpret_cast<int *>(base + off_ids);
    auto *so = reinterpret_cast<long long *>(base + off_so);
    cuda_check(cudaMemsetAsync(h, 0, sizeof(StaticHeader), s), "memset");
    static_prep_kernel<<<1, kPrepThreads, 0, s>>>(n, node_off, total_nodes, kPatternNodeTile, h, ids, so);
    const long long cells = (long long)(g.L + 1) * g.X * g.Y;
    static_check_kernel<<<std::min(1184, (n + 255) / 256), 256, 0, s>>>(n, node_off, nodes, par, route_off,
                                                                        route_cap, routes_len, cells, h);
    cuda_check(cudaGetLastError(), "launch");
    StaticHeader hh{};
    cuda_check(cudaMemcpyAsync(&hh, h, sizeof hh, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (hh.status & kBadOffsets)
        throw Error(ERR_INVALID, "node_off must start at 0, end at total_nodes and give every tree a node (near net " +
                                     std::to_string(hh.bad_net) + ")");
    if (hh.status & kBadRecord)
        throw Error(ERR_INVALID, "route record of net " + std::to_string(hh.bad_net) + " lies outside routes");
    if (hh.status & kBadNode)
        throw Error(ERR_INVALID, "node position out of range (net " + std::to_string(hh.bad_net) + ")");
    if (hh.status & kBadParent)
        throw Error(ERR_STATE, "tree nodes must be in preorder with par[i] < i (net " + std::to_string(hh.bad_net) + ")");
    const size_t need = off_tab + sizeof(double) * (size_t)pattern_scratch_doubles(hh.big_nodes);
    if (need > kStaticScratchBytes)
        throw Error(ERR_CAPACITY, "batch needs " + std::to_string(need) + " bytes of scratch (" +
                                      std::to_string(hh.big_nodes) + " nodes in nets of more than " +
                                      std::to_string(kPatternNodeTile) + " nodes); the static scratch holds " +
                                      std::to_string(kStaticScratchBytes) + " bytes");
    TreeBatchDev tb{ids, node_off, nodes, par, route_off, route_cap, routes,
                    reinterpret_cast<double *>(base + off_tab), reinterpret_cast<const int64_t *>(so),
                    hh.big_nodes, n};
    tb.queue = &h->queue;
    tb.tile = kPatternNodeTile;
    launch_pattern_route(g, tb, stamp, s);
    cuda_check(cudaGetLastError(), "launch");
}

}  // namespace igr
