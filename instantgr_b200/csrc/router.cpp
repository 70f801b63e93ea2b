// Rip-up-and-reroute driver (src/main.cpp:22-73, src/Lshape_route.hpp:155-257,
// src/Lshape_route_detour.hpp:726-1112), restated for one GPU:
//
//   open      read, pin selection, Steiner trees, split (host threads); trees
//             and conflict shapes uploaded once and kept resident
//   phase 1   HPWL order -> GPU colouring -> per batch: cost refresh, tree DP,
//             wire commit, via commit
//   pass i    overflow marking -> congestion view -> detour DAGs of the marked
//             nets (host threads) -> GPU colouring -> per batch: rip-up, cost
//             refresh, DAG DP, wire commit, via commit
//
// InstantGR runs one pass; rrr_iters > 1 repeats the pass on the nets that
// still overflow.  All per-batch work is stream-ordered with no host
// synchronisation between batches (the reference synchronises after every
// phase-2 launch), and no device memory is allocated per run once the
// buffers have grown to the design's size.
#include "router.hpp"
#include "seed_model.hpp"
#include "hooks.hpp"

#include <dlfcn.h>
#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <map>
#include <mutex>
#include <numeric>
#include <thread>

namespace igr {

void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw Error(ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ device memory cache
namespace {
std::mutex g_cache_mu;
std::map<std::pair<int, size_t>, std::vector<void *>> g_cache;  // (device, block bytes) -> free blocks
std::atomic<long long> g_mallocs{0}, g_malloc_us{0}, g_trims{0};  // cudaMalloc calls and their time, trims

size_t block_bytes(size_t bytes) {
    const size_t g = bytes >= (size_t(1) << 20) ? (size_t(2) << 20) : 512;  // 2 MiB granules for large blocks
    return (bytes + g - 1) / g * g;
}
}  // namespace

void *dev_alloc(size_t bytes) {
    const size_t b = block_bytes(bytes);
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        // smallest cached block that fits and wastes at most half of itself
        auto it = g_cache.lower_bound({dev, b});
        if (it != g_cache.end() && it->first.first == dev && it->first.second <= 2 * b && !it->second.empty()) {
            void *p = it->second.back();
            it->second.pop_back();
            if (it->second.empty()) g_cache.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaMalloc(&p, b) != cudaSuccess) {
        cudaGetLastError();
        dev_trim();
        g_trims++;
        cuda_check(cudaMalloc(&p, b), "cudaMalloc");
    }
    g_mallocs++;
    g_malloc_us += std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
    return p;
}

void dev_alloc_stats(long long *mallocs, long long *us, long long *trims) {
    *mallocs = g_mallocs.load();
    *us = g_malloc_us.load();
    *trims = g_trims.load();
}

void dev_free(void *p, size_t bytes) {
    if (!p) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    std::lock_guard<std::mutex> lock(g_cache_mu);
    g_cache[{dev, block_bytes(bytes)}].push_back(p);
}

void dev_trim() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (auto it = g_cache.begin(); it != g_cache.end();) {
        if (it->first.first != dev) { ++it; continue; }
        for (void *p : it->second) cudaFree(p);
        it = g_cache.erase(it);
    }
}

namespace {
std::mutex g_pinned_mu;
std::map<size_t, std::vector<void *>> g_pinned;  // block bytes -> free page-locked blocks
}  // namespace

void *pinned_alloc(size_t bytes) {
    const size_t b = block_bytes(bytes);
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        auto it = g_pinned.lower_bound(b);
        if (it != g_pinned.end() && it->first <= 2 * b && !it->second.empty()) {
            void *p = it->second.back();
            it->second.pop_back();
            if (it->second.empty()) g_pinned.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    cuda_check(cudaMallocHost(&p, b), "cudaMallocHost");
    return p;
}

bool pinned_cached(size_t bytes) {
    const size_t b = block_bytes(bytes);
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    auto it = g_pinned.lower_bound(b);
    return it != g_pinned.end() && it->first <= 2 * b && !it->second.empty();
}

void pinned_free(void *p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned[block_bytes(bytes)].push_back(p);
}

// True when this process has initialised the CUDA driver already, found
// without initialising it: cuCtxGetCurrent of an already loaded driver
// library answers CUDA_ERROR_NOT_INITIALIZED (3) before cuInit.
bool cuda_driver_ready() {
    void *h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_NOLOAD);
    if (!h) return false;
    using GetCurrent = int (*)(void **);
    auto f = reinterpret_cast<GetCurrent>(dlsym(h, "cuCtxGetCurrent"));
    void *ctx = nullptr;
    const bool ready = f && f(&ctx) == 0;
    dlclose(h);
    return ready;
}

namespace {
// host staging array without value initialisation, in cached page-locked
// memory (uploads at full speed; pages reused by the next pass)
template <typename T>
struct HostArray {
    T *p = nullptr;
    size_t n = 0;
    explicit HostArray(size_t count) : p(static_cast<T *>(pinned_alloc((count ? count : 1) * sizeof(T)))), n(count) {}
    ~HostArray() { pinned_free(p, (n ? n : 1) * sizeof(T)); }
    HostArray(const HostArray &) = delete;
    HostArray &operator=(const HostArray &) = delete;
    T *data() { return p; }
    const T *data() const { return p; }
    size_t size() const { return n; }
    T &operator[](size_t i) { return p[i]; }
    const T &operator[](size_t i) const { return p[i]; }
    T *begin() { return p; }
};
}  // namespace

// ------------------------------------------------------------------ grid
void GridOwner::create(int L, int X, int Y, int DIR, const int *xl, const int *yl, double unit_wire,
                       double unit_via, const double *sc, const float *cap_ref, cudaStream_t s) {
    if (L != kRouteLayers) throw Error(ERR_INVALID, "the router handles 9 routing layers");
    if (X < 2 || Y < 2) throw Error(ERR_INVALID, "grid must be at least 2x2");
    if (X > kMaxTrackCells || Y > kMaxTrackCells)
        throw Error(ERR_CAPACITY, "tracks longer than 15360 GCells are not supported (the reference's limit)");
    g = GridDev();
    g.L = L; g.X = X; g.Y = Y; g.DIR = DIR;
    g.N = (int64_t)L * X * Y;
    layer_first.assign(L + 1, 0);
    for (int l = 0; l < L; l++) layer_first[l + 1] = layer_first[l] + ((((l & 1) ^ DIR) != 0) ? X : Y);
    g.ntracks = layer_first[L];
    g.unit_wire = unit_wire;
    g.unit_via = unit_via;
    cap.alloc(g.N); demand.alloc(g.N); vcost.alloc(g.N); presum.alloc(g.N);
    pre.alloc(g.N); stamp.alloc(g.N);
    xlen.upload(xl, X - 1, s); ylen.upload(yl, Y - 1, s);
    short_cost.upload(sc, L, s);
    dirty_cost.alloc(g.ntracks); dirty_commit.alloc(g.ntracks);
    stats.alloc(kStatSlots); err.alloc(1);
    score.alloc(g.ntracks + 1);
    g.cap = cap.p; g.demand = demand.p; g.vcost = vcost.p; g.presum = presum.p;
    g.pre = pre.p; g.stamp = stamp.p; g.xlen = xlen.p; g.ylen = ylen.p; g.short_cost = short_cost.p;
    g.dirty_cost = dirty_cost.p; g.dirty_commit = dirty_commit.p; g.stats = stats.p; g.err = err.p;
    // capacity: reference layout -> track layout through a staging buffer
    DevBuf<float> tmp;
    tmp.upload(cap_ref, g.N, s);
    launch_to_track_layout(g, tmp.p, cap.p, s);
    cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(vcost.p, 0, g.N * sizeof(float), s), "memset");
    cuda_check(cudaMemsetAsync(presum.p, 0, g.N * sizeof(double), s), "memset");
    reset_demand(s);
    cuda_check(cudaStreamSynchronize(s), "create");
}

void GridOwner::reset_demand(cudaStream_t s) {
    cuda_check(cudaMemsetAsync(demand.p, 0, g.N * sizeof(float), s), "memset");
    cuda_check(cudaMemsetAsync(pre.p, 0, g.N * sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(stamp.p, 0, g.N * sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(stats.p, 0, kStatSlots * sizeof(unsigned long long), s), "memset");
    cuda_check(cudaMemsetAsync(dirty_commit.p, 0, g.ntracks, s), "memset");
    mark_all_dirty(s);
}

void GridOwner::mark_all_dirty(cudaStream_t s) {
    cuda_check(cudaMemsetAsync(dirty_cost.p, 1, g.ntracks, s), "memset");
}

int GridOwner::check_error(cudaStream_t s) {
    int e = 0;
    cuda_check(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (e) cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    return e;
}

// ------------------------------------------------------------------ kernel timer
void KernelTimer::begin(int k) {
    if (!on) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    ev[k].push_back({a, b});
}
void KernelTimer::end(int k) {
    if (!on) return;
    cudaEventRecord(ev[k].back().second, s);
    launches[k]++;
}
void KernelTimer::collect() {
    for (int k = 0; k < KC_N; k++) {
        for (auto &p : ev[k]) {
            float t = 0;
            if (cudaEventElapsedTime(&t, p.first, p.second) == cudaSuccess) ms[k] += t;
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        ev[k].clear();
    }
}
void KernelTimer::reset() {
    collect();
    for (int k = 0; k < KC_N; k++) { ms[k] = 0; launches[k] = 0; }
}

void ShapeDev::upload(const ShapeSet &sh, int X, int Y, int sp, cudaStream_t st, int threads) {
    pt_n.release();  // whole ranges: host-built lists are used as they are
    claim_n.release();
    pt_off.upload(sh.pt_off, st); pts.upload(sh.pts, st); pt_net.upload(sh.pt_net, st);
    h_off.upload(sh.h_off, st); hseg.upload(sh.hseg, st);
    v_off.upload(sh.v_off, st); vseg.upload(sh.vseg, st);
    npts = (int)sh.pts.size();
    nshapes = (int)sh.pt_off.size() - 1;
    sparsity = sp;
    std::vector<int> co, cl;
    build_claims(nshapes, sh.pt_off.data(), sh.pts.data(), sh.h_off.data(), sh.hseg.data(), sh.v_off.data(),
                 sh.vseg.data(), X, Y, sp, co, cl, threads);
    claim_off.upload(co, st);
    claim.upload(cl, st);
    cuda_check(cudaStreamSynchronize(st), "claims");  // host vectors go out of scope
    bytes = 4 * (int64_t)(sh.pt_off.size() + 2 * sh.pts.size() + sh.h_off.size() + sh.hseg.size() +
                          sh.v_off.size() + sh.vseg.size() + co.size() + cl.size());
}

// ------------------------------------------------------------------ router
Router::~Router() {
    if (grid_thread.joinable()) grid_thread.join();
    if (dt_packing.valid()) dt_packing.wait();
    if (order1_pending.valid()) order1_pending.wait();
    if (s) cudaStreamSynchronize(s);  // no copy from a page-locked buffer is in flight below
    kt.collect();
    if (graph1_exec) cudaGraphExecDestroy(graph1_exec);
    if (ev0) cudaEventDestroy(ev0);
    for (int i = 0; i < 2; i++) {
        if (ev_join[i]) cudaEventDestroy(ev_join[i]);
        if (s_cls[i]) cudaStreamDestroy(s_cls[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_gfork) cudaEventDestroy(ev_gfork);
    if (ev_gjoin) cudaEventDestroy(ev_gjoin);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
    // The host copy of the design and its routing nets (tens of ms of frees on
    // the 800k-net design) goes on a thread of its own, beside whatever the
    // caller does next; the nets' arenas return to a block cache that is never
    // destroyed, so the frees may also outlast the program's static objects.
    try {
        auto host = std::make_unique<std::pair<Design, NetSet>>(std::move(d), std::move(ns));
        std::thread([h = std::move(host)]() mutable { h.reset(); }).detach();
    } catch (...) {
        // no thread: the members are freed here, as they would be otherwise
    }
}

void Router::open(const char *cap, const char *net) {
    const double t0 = now_s();
    // The CUDA driver, the caller's device context and the routing grid are
    // brought up on a side thread while the host parses and builds trees (the
    // first CUDA call of a process can take a second).  The device is the
    // calling thread's current one; before the driver is initialised no thread
    // can have chosen one, so it is the runtime's default, device 0.
    int dev = 0;
    if (cuda_driver_ready() && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    std::promise<bool> cap_read;  // true: the capacities are parsed; false: open failed
    std::future<bool> cap_ok = cap_read.get_future();
    grid_thread = std::thread([this, dev, f = std::move(cap_ok)]() mutable {
        try {
            const double c0 = now_s();
            cuda_check(cudaSetDevice(dev), "cudaSetDevice");
            cuda_check(cudaFree(nullptr), "device context");
            ctx_seconds = now_s() - c0;
            if (f.get()) create_grid();
        } catch (...) {
            grid_err = std::current_exception();
        }
    });
    try {
        read_design(d, cap, net, threads);
    } catch (...) {
        cap_read.set_value(false);
        throw;
    }
    cap_read.set_value(true);
    const double t_read = now_s();
    build_netset(d, ns, threads);
    const double t_nets = now_s();
    const int R = (int)ns.nets.size();
    // phase-1 routing priority: HPWL, largest first (Lshape_route.hpp:170-172),
    // with the reference's (unstable) std::sort and comparator: (key, id)
    // pairs compared on the key alone take the same sequence of comparisons
    // and moves, hence give the same order, as the ids compared through the
    // nets.  Sorted on a host thread while the trees are laid out and the
    // device is set up; the keys stay for the rip-up order of the reroute passes
    hpwl_keys.resize(R);
    parallel_for(R, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) hpwl_keys[i] = ns.nets[i].hpwl;
    });
    order1_pending = std::async(std::launch::async, [this, R] {
        std::vector<std::pair<int, int>> kv(R);
        for (int i = 0; i < R; i++) kv[i] = {hpwl_keys[i], i};
        std::sort(kv.begin(), kv.end(),
                  [](const std::pair<int, int> &l, const std::pair<int, int> &r) { return l.first > r.first; });
        std::vector<int> order(R);
        for (int i = 0; i < R; i++) order[i] = kv[i].second;
        return order;
    });
    // trees in DFS preorder, net-id order, and the phase-1 route record layout:
    // the nets' sizes and record capacities read in parallel, then the prefix
    // sums over plain arrays
    tree_off.assign(R + 1, 0);
    route_cap.assign(R, 0);
    parallel_for(R, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) {
            const auto &n = ns.nets[i];
            tree_off[i + 1] = (int)n.tnode.size();
            route_cap[i] = (int)std::max<int64_t>(12 * (int64_t)n.pins.size(), 8 * (int64_t)n.tnode.size() + 1);
        }
    });
    for (int i = 0; i < R; i++) tree_off[i + 1] += tree_off[i];
    tree_nodes.resize(tree_off[R]);
    tree_par.resize(tree_off[R]);
    // algorithmic bytes of one phase-1 tree DP pass: per node the 8 via-column
    // costs (f32); per straight edge 9 layers x 2 presum values (f64); per bent
    // edge 18 legs x 2 presum values and the two corner via columns (9 x f32 each)
    std::vector<int64_t> net_bytes(R);
    parallel_for(R, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) {
            const int a = tree_off[i], m = tree_off[i + 1] - a;
            flatten_tree(ns.nets[i], tree_nodes.data() + a, tree_par.data() + a);
            int64_t nb = 32 * (int64_t)m;
            for (int j = 1; j < m; j++) {
                const int p = tree_par[a + j];
                if (p < 0 || p >= j) continue;
                const int v = tree_nodes[a + j], pv = tree_nodes[a + p];
                const int x = v / ns.Y % ns.X, y = v % ns.Y, px = pv / ns.Y % ns.X, py = pv % ns.Y;
                nb += (x == px || y == py) ? 144 : 360;
            }
            net_bytes[i] = nb;
        }
    });
    route_off.assign(R, 0);
    route_end1 = 0;
    scratch_off.assign(R, -1);
    scratch_nodes = 0;
    int64_t dpb = 0;
    for (int i = 0; i < R; i++) {
        route_off[i] = route_end1;
        route_end1 += route_cap[i];
        const int cnt = tree_off[i + 1] - tree_off[i];
        if (cnt > kPatternNodeTile) { scratch_off[i] = scratch_nodes; scratch_nodes += cnt; }
        dpb += net_bytes[i];
    }
    route_off1 = route_off;
    route_cap1 = route_cap;
    dp_bytes = (double)dpb;
    if (verbose)
        std::fprintf(stderr, "[igr] read+trees %.2fs (read %.3f, pins+trees %.3f, layout %.3f): %d nets, %d routing nets\n",
                     now_s() - t0, t_read - t0, t_nets - t_read, now_s() - t_nets, d.num_nets(), R);
}

// Device state is created and the inputs uploaded on the first run, so that
// opening a design (parsing, pin selection, trees) needs no GPU.
void Router::create_grid() {
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < 2; i++) {
        cuda_check(cudaStreamCreateWithFlags(&s_cls[i], cudaStreamNonBlocking), "stream");
        cuda_check(cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming), "event");
    }
    cuda_check(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming), "event");
    cuda_check(cudaEventCreateWithFlags(&ev_gfork, cudaEventDisableTiming), "event");
    cuda_check(cudaEventCreateWithFlags(&ev_gjoin, cudaEventDisableTiming), "event");
    cuda_check(cudaEventCreate(&ev0), "event");
    cuda_check(cudaEventCreate(&ev1), "event");
    const int L = d.L - 1, X = d.X, Y = d.Y;
    std::vector<double> sc(L);
    for (int l = 0; l < L; l++) sc[l] = d.short_cost[l + 1];
    // routing layers are file layers 1..L, contiguous in d.cap
    go.create(L, X, Y, d.layer_dir[1], d.x_edge_len.data(), d.y_edge_len.data(), d.unit_wire, d.unit_via, sc.data(),
              d.cap.data() + (size_t)X * Y, s);
    grid_ready = true;
}

void Router::join_grid() {
    if (grid_thread.joinable()) grid_thread.join();
    if (grid_err) {
        std::exception_ptr e = grid_err;
        grid_err = nullptr;
        std::rethrow_exception(e);
    }
}

// Conflict shapes and claim lists on the device (shapes.cu): counts and
// offsets, the totals to the host for the allocation, then the fill.
void Router::device_shapes(const ShapeArgs &a, ShapeDev &sd) {
    sd.pt_off.alloc((size_t)a.n + 1);
    sd.claim_off.alloc((size_t)a.n + 1);
    d_shape_tot.alloc(2);
    const double t0 = now_s();
    launch_shape_count(a, sd.pt_off.p, sd.claim_off.p, d_shape_tot.p, s);
    long long h_tot[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(h_tot, d_shape_tot.p, sizeof h_tot, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "shape counts");
    const double t1 = now_s();
    if (h_tot[0] > INT32_MAX || h_tot[1] > INT32_MAX) throw Error(ERR_CAPACITY, "conflict shapes exceed 32-bit offsets");
    sd.pts.alloc((size_t)h_tot[0]);
    sd.claim.alloc((size_t)h_tot[1]);
    if (test_hooks().shape_dedupe.load()) {
        sd.pt_n.alloc((size_t)std::max(a.n, 1));
        sd.claim_n.alloc((size_t)std::max(a.n, 1));
    } else {
        sd.pt_n.release();
        sd.claim_n.release();
    }
    launch_shape_fill(a, sd.pt_off.p, sd.claim_off.p, sd.pts.p, sd.claim.p, sd.pt_n.p, sd.claim_n.p, s);
    if (verbose) {
        long long m = 0, us = 0, tr = 0;
        dev_alloc_stats(&m, &us, &tr);
        std::fprintf(stderr,
                     "[igr] conflict shapes of %d nets: counts %.4f s, allocations and fill launch %.4f s "
                     "(cudaMalloc so far: %lld calls, %.3f s, %lld trims)\n",
                     a.n, t1 - t0, now_s() - t1, m, us * 1e-6, tr);
    }
    sd.npts = (int)h_tot[0];
    sd.nshapes = a.n;
    sd.sparsity = a.sparsity;
    sd.bytes = 0;
}

void Router::ensure_device() {
    if (device_ready) return;
    const double t0 = now_s();
    join_grid();
    if (!grid_ready) create_grid();
    const int L = d.L - 1, X = d.X, Y = d.Y;
    const double t_grid = now_s();
    // resident inputs
    d_tree_off.upload(tree_off, s);
    d_tree_nodes.upload(tree_nodes.data(), tree_nodes.size(), s);
    d_tree_par.upload(tree_par.data(), tree_par.size(), s);
    d_scratch_off.upload(scratch_off, s);
    d_scratch.alloc((size_t)pattern_scratch_doubles(scratch_nodes));
    d_vcnt.alloc((size_t)go.g.N);
    cuda_check(cudaMemsetAsync(d_vcnt.p, 0, (size_t)go.g.N * sizeof(int), s), "memset");
    d_route_off1.upload(route_off1, s);
    d_route_cap1.upload(route_cap1, s);
    d_route_off.alloc(route_off1.size());
    d_route_cap.alloc(route_cap1.size());
    const double t_trees = now_s();
    const int R = (int)ns.nets.size();
    {
        // phase-1 conflict shapes and claim lists from the resident trees; phase 1
        // samples every 15th segment cell (database_cuda.hpp:439)
        ShapeArgs a;
        a.tree_off = d_tree_off.p; a.tree_nodes = d_tree_nodes.p; a.tree_par = d_tree_par.p;
        a.n = R; a.X = X; a.Y = Y; a.sparsity = 15;
        device_shapes(a, d_shapes1);
    }
    const double t_shapes = now_s();
    const double t_claims = t_shapes;
    // phase-1 colouring ranks: the reversed routing priority (the last rank wins conflicts)
    if (order1_pending.valid()) order1 = order1_pending.get();
    std::vector<int> perm1(order1.rbegin(), order1.rend());
    d_perm1.upload(perm1, s);
    std::vector<int> ids(R);
    std::iota(ids.begin(), ids.end(), 0);
    d_all_ids.upload(ids, s);
    // host-to-device bytes of the setup: grid, trees, record layout, conflict shapes, ranks
    setup_h2d = (int64_t)go.g.N * 4 + 4 * (int64_t)(X + Y - 2) + 8 * L + 4 * (int64_t)tree_off.size() +
                8 * (int64_t)tree_nodes.size() + 8 * (int64_t)scratch_off.size() + 12 * (int64_t)R + 8 * (int64_t)R;
    cuda_check(cudaStreamSynchronize(s), "inputs");
    device_ready = true;
    if (verbose)
        std::fprintf(stderr,
                     "[igr] device setup %.3fs (waiting for the context and grid %.3f, trees %.3f, shapes and claims "
                     "%.3f, rest %.3f; the context took %.3f on the side thread)\n",
                     now_s() - t0, t_grid - t0, t_trees - t_grid, t_shapes - t_trees, now_s() - t_claims, ctx_seconds);
}

// Grows the route buffer to `need` ints, keeping the records already written.
// The first buffer leaves 40% room for the records the rip-up passes append
// (on the 800k-net design three passes append about 30% of the phase-1
// records), so that a pass rarely has to grow it.
void Router::grow_routes(int64_t need) {
    if ((int64_t)routes.n >= need) return;
    DevBuf<int> nb;
    nb.alloc((size_t)std::max<int64_t>(need + (routes.n ? 0 : need * 2 / 5), (int64_t)(routes.n * 3 / 2)));
    if (routes.p && routes.n > 0)
        cuda_check(cudaMemcpyAsync(nb.p, routes.p, routes.n * sizeof(int), cudaMemcpyDeviceToDevice, s), "D2D");
    std::swap(routes.p, nb.p);
    std::swap(routes.n, nb.n);
}

void Router::run() {
    if (!seed || seed_mode == 0) {
        run_once(false);
        return;
    }
    // scores are the evaluator's totals, computed on the device
    auto total = [&] {
        double v[4];
        evaluate(v, nullptr);
        return v[3];
    };
    if (seed_mode == 1) {
        // nothing is decided on the score: it is computed when asked for
        run_once(true);
        seed_used = true;
        seed_score_due = true;
        return;
    }
    seed_score_due = false;
    // seeded run judged against the plain run: the better total score is kept
    const double t0 = now_s();
    run_once(true);
    const double seeded_score = total();
    RouteBackup bk;
    save_result(bk);
    run_once(false);
    const double plain_score = total();
    seed_used = seeded_score < plain_score;
    if (seed_used) restore_result(bk);
    seed_scores[0] = plain_score;
    seed_scores[1] = seeded_score;
    st.wall = now_s() - t0;
    if (verbose)
        std::fprintf(stderr, "[igr] seeded %.0f vs plain %.0f: %s result kept\n", seeded_score, plain_score,
                     seed_used ? "seeded" : "plain");
}

// Seed statistics of the last run (igr_router_seed_stats); a seeded-only
// run's score is the evaluator's total of its result, computed on the first
// request.
void Router::seed_stats(double out[4]) {
    if (seed_score_due) {
        double v[4];
        evaluate(v, nullptr);
        seed_scores[1] = v[3];
        seed_score_due = false;
    }
    out[0] = seed_used ? 1.0 : 0.0;
    out[1] = seed_scores[1];
    out[2] = seed_scores[0];
    out[3] = seed_ms;
}

void Router::save_result(RouteBackup &b) {
    b.routes.alloc(std::max<size_t>(1, (size_t)route_end));
    if (route_end)
        cuda_check(cudaMemcpyAsync(b.routes.p, routes.p, route_end * sizeof(int), cudaMemcpyDeviceToDevice, s), "D2D");
    b.demand.alloc(go.g.N);
    cuda_check(cudaMemcpyAsync(b.demand.p, go.demand.p, go.g.N * sizeof(float), cudaMemcpyDeviceToDevice, s), "D2D");
    cuda_check(cudaStreamSynchronize(s), "backup");
    b.route_off = route_off;
    b.route_cap = route_cap;
    b.route_end = route_end;
    b.st = st;
    b.kt_ms.assign(kt.ms, kt.ms + KC_N);
    b.score[0] = score_wl;
    b.score[1] = score_via;
    b.score[2] = score_of;
    b.cost_cells = cost_cells;
    b.commit_cells = commit_cells;
    b.commit_refresh_cells = commit_refresh_cells;
    b.color_bytes = color_bytes;
}

void Router::restore_result(RouteBackup &b) {
    grow_routes(b.route_end);
    if (b.route_end)
        cuda_check(cudaMemcpyAsync(routes.p, b.routes.p, b.route_end * sizeof(int), cudaMemcpyDeviceToDevice, s), "D2D");
    cuda_check(cudaMemcpyAsync(go.demand.p, b.demand.p, go.g.N * sizeof(float), cudaMemcpyDeviceToDevice, s), "D2D");
    cuda_check(cudaStreamSynchronize(s), "restore");
    route_off = b.route_off;
    route_cap = b.route_cap;
    route_end = b.route_end;
    d_route_off.upload(route_off, s);  // the device's offsets follow the host's
    d_route_cap.upload(route_cap, s);
    st = b.st;
    score_wl = b.score[0];
    score_via = b.score[1];
    score_of = b.score[2];
    cost_cells = b.cost_cells;
    commit_cells = b.commit_cells;
    commit_refresh_cells = b.commit_refresh_cells;
    color_bytes = b.color_bytes;
    h_routes_valid = false;
    go.mark_all_dirty(s);
}

// Prediction of the attached congestion seed for this design (once), the
// seed demand in the track layout and the predicted overflow per GCell.
void Router::device_seed_features(DevBuf<__nv_bfloat16> &feat, cudaStream_t st) {
    ensure_device();
    const int X = go.g.X, Y = go.g.Y;
    const size_t XY = (size_t)X * Y, D = (size_t)(X + 1) * (Y + 1);
    DevBuf<float> cap0;
    DevBuf<int> pins;
    DevBuf<long long> dh, dv;
    cap0.upload(d.cap.data(), XY, st);  // file layer 0
    pins.alloc(XY);
    dh.alloc(D);
    dv.alloc(D);
    feat.alloc(XY * 16);
    // the trees were uploaded on the router's stream
    cuda_check(cudaStreamSynchronize(s), "trees");
    launch_seed_features(go.g, (int)ns.nets.size(), d_tree_off.p, d_tree_nodes.p, cap0.p, d.L, pins.p, dh.p, dv.p,
                         feat.p, st);
    cuda_check(cudaGetLastError(), "seed features");
    cuda_check(cudaStreamSynchronize(st), "seed features");
}

void Router::prepare_seed() {
    if (seed_ready) return;
    const double t0 = now_s();
    const int L = go.g.L, X = go.g.X, Y = go.g.Y;
    const size_t nf = (size_t)X * Y * 16;
    DevBuf<__nv_bfloat16> feat;
    device_seed_features(feat, seed->s);
    const double t1 = now_s();
    DevBuf<float> pred, ref, cap;
    pred.alloc(nf);
    cuda_check(cudaMemsetAsync(pred.p, 0, nf * sizeof(float), seed->s), "memset");
    seed->predict(X, Y, feat.p, pred.p);
    const double t2 = now_s();
    cap.alloc((size_t)L * X * Y);
    launch_from_track_layout_f(go.g, go.cap.p, cap.p, seed->s);
    ref.alloc((size_t)L * X * Y);
    launch_seed_demand(X, Y, L, pred.p, (float)seed_alpha, seed_kind, cap.p, ref.p, seed->s);
    DevBuf<float> over;
    over.alloc((size_t)X * Y);
    launch_seed_overflow(X, Y, L, pred.p, cap.p, over.p, seed->s);
    std::vector<float> ov((size_t)X * Y);
    cuda_check(cudaMemcpyAsync(ov.data(), over.p, ov.size() * 4, cudaMemcpyDeviceToHost, seed->s), "D2H");
    cuda_check(cudaStreamSynchronize(seed->s), "seed");
    d_seed_dem.alloc(go.g.N);
    launch_to_track_layout(go.g, ref.p, d_seed_dem.p, s);
    d_seed_cur.alloc(go.g.N);
    cuda_check(cudaMemsetAsync(d_seed_cur.p, 0, go.g.N * sizeof(float), s), "memset");
    // summed-area table of the predicted overflow for the rip-up order
    seed_sat.assign((size_t)(X + 1) * (Y + 1), 0.0);
    for (int x = 0; x < X; x++)
        for (int y = 0; y < Y; y++)
            seed_sat[(size_t)(x + 1) * (Y + 1) + y + 1] = ov[(size_t)x * Y + y] + seed_sat[(size_t)x * (Y + 1) + y + 1] +
                                                          seed_sat[(size_t)(x + 1) * (Y + 1) + y] -
                                                          seed_sat[(size_t)x * (Y + 1) + y];
    cuda_check(cudaStreamSynchronize(s), "seed");
    seed_ready = true;
    seed_ms = 1e3 * (now_s() - t0);
    if (verbose)
        std::fprintf(stderr, "[igr] congestion seed: %.1f ms (features %.1f, network %.1f)\n", seed_ms,
                     1e3 * (t1 - t0), 1e3 * (t2 - t1));
}

// Starts the seed of a phase-1 pass on freshly reset demand: constant seeds are
// added at once, shrinking ones by the first step of the batch loop.
void Router::seed_begin() {
    if (!seed_active) return;
    cuda_check(cudaMemsetAsync(d_seed_cur.p, 0, go.g.N * sizeof(float), s), "memset");
    if (seed_levels == 0) launch_seed_step(go.g.N, go.demand.p, d_seed_dem.p, d_seed_cur.p, 1.f, s);
}

// predicted overflow per GCell over a net's bounding box
double Router::seed_pressure(int net) const {
    const RNet &n = ns.nets[net];
    const int Y1 = ns.Y + 1;
    auto at = [&](int x, int y) { return seed_sat[(size_t)x * Y1 + y]; };
    const double s = at(n.maxx + 1, n.maxy + 1) - at(n.minx, n.maxy + 1) - at(n.maxx + 1, n.miny) + at(n.minx, n.miny);
    return s / ((double)(n.maxx - n.minx + 1) * (n.maxy - n.miny + 1));
}

void Router::run_once(bool seeded) {
    ensure_device();
    cudaGetLastError();  // start from a clean error state
    if (seeded) prepare_seed();
    seed_active = seeded;
    const double t0 = now_s();
    st = RouterStats();
    kt.s = s;
    kt.reset();
    go.reset_demand(s);
    cuda_check(cudaMemsetAsync(d_vcnt.p, 0, (size_t)go.g.N * sizeof(int), s), "memset");
    d_cops.alloc(5);
    cuda_check(cudaMemsetAsync(d_cops.p, 0, 5 * sizeof(unsigned long long), s), "memset");
    global_stamp = 0;
    h_routes_valid = false;
    const int R = (int)ns.nets.size();
    // phase-1 records at their fixed offsets; reroutes are appended after them
    route_off = route_off1;
    route_cap = route_cap1;
    route_end = route_end1;
    int m = mode;
    if (m < 0) m = R > 20000000 ? 2 : (R > 5000000 ? 1 : 0);
    mode_eff = m;
    // the device DAG builder of the first reroute pass needs every net's tree in
    // adjacency order: packed on a side thread while phase 1 keeps the device busy
    if (!dt_ready && !dt_packing.valid() && rrr_iters > 0 && !host_dags)
        dt_packing = std::async(std::launch::async, [this] { pack_dag_trees(); });
    // the seed demand steers phase 1 only (added in phase1()) and is taken out before rip-up
    phase1();
    if (seeded) {
        launch_seed_step(go.g.N, go.demand.p, d_seed_dem.p, d_seed_cur.p, 0.f, s);
        go.mark_all_dirty(s);
    }
    for (int it = 0; it < rrr_iters; it++)
        if (!rrr_pass(it)) break;
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (int e = go.check_error(s)) throw Error(e, "device error during routing");
    st.wall = now_s() - t0;
    kt.collect();
    compute_score();
    ran = true;
    if (verbose)
        std::fprintf(stderr, "[igr] route %.3fs  WL %.0f  via %.0f  OF %.0f  total %.0f\n", st.wall, score_wl,
                     score_via, score_of, score_wl + score_via + score_of);
}

void Router::fetch_routes() {
    if (h_routes_valid) return;
    const int R = (int)route_off.size();
    h_route_at.assign((size_t)R + 1, 0);
    if (route_end == 0 || R == 0) {
        h_routes_ptr = nullptr;
        h_routes_valid = true;
        return;
    }
    // Records sit at offsets with room for their largest size, and each
    // rip-up pass appends new ones: pack the live records on the device
    // (lengths, scan, copy) and bring only those and their offsets back.  The
    // device holds the record offsets already (every pass brings them up to
    // date there).
    d_dense_off.alloc((size_t)R + 1);
    launch_record_offsets(routes.p, d_route_off.p, R, route_end, d_dense_off.p, s);
    cuda_check(cudaMemcpyAsync(h_route_at.data(), d_dense_off.p, ((size_t)R + 1) * 8, cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    const int64_t live = h_route_at[R];
    d_dense.alloc((size_t)live);
    launch_record_copy(routes.p, d_route_off.p, R, d_dense_off.p, d_dense.p, s);
    // Page-locked memory copies fastest, but locking a very large new block
    // costs more than the copy it speeds up: a first copy of more than 512 MB
    // goes to pageable memory.  Smaller blocks are locked once and, given back
    // to the process-wide cache when the router closes, serve the next ones.
    const size_t bytes = (size_t)live * sizeof(int);
    if (bytes <= ((size_t)512 << 20) || (h_routes.p && h_routes.n >= (size_t)live) || pinned_cached(bytes)) {
        h_routes.alloc((size_t)live);
        h_routes_ptr = h_routes.p;
    } else {
        h_routes_pageable.resize((size_t)live);
        h_routes_ptr = h_routes_pageable.data();
    }
    cuda_check(cudaMemcpyAsync(const_cast<int *>(h_routes_ptr), d_dense.p, bytes, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (bytes > ((size_t)256 << 20)) d_dense.release();  // a large packed copy gives its HBM back
    st.d2h_bytes += (int64_t)bytes + ((int64_t)R + 1) * 8;
    st.launches += 3;
    h_routes_valid = true;
}

// Phase 1 (Lshape_route.hpp:155-257)
// Routing order of phase 1 from the colouring.  Plain form: each batch in
// colouring order, one DP launch.  Batched form: inside each batch the nets
// are split into size classes (results do not depend on the order of nets
// within a batch): large nets (global scratch) first, then medium, then small,
// each by node count, largest first; one DP launch per class.
void Router::plan_phase1(int nb, std::vector<int> &batch_off, std::vector<int> &class_off) {
    const int R = (int)ns.nets.size();
    PlanArgs pa;
    pa.n = R; pa.nb = nb; pa.bat = d_bat.p; pa.perm = d_perm1.p; pa.node_off = d_tree_off.p;
    pa.classes = batched ? tune.classes : 1;
    pa.split = tune.split;
    pa.big = kPatternNodeTile;
    d_plan_hist.alloc((size_t)plan_hist_size(nb));
    d_plan_offs.alloc(3 * (size_t)nb + 1);
    d_ids.alloc(R);
    launch_plan(pa, d_plan_hist.p, d_ids.p, d_plan_offs.p, go.g.err, s);
    st.launches += 3;
    std::vector<int> offs(3 * (size_t)nb + 1);
    cuda_check(cudaMemcpyAsync(offs.data(), d_plan_offs.p, offs.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "plan");
    st.d2h_bytes += (int64_t)offs.size() * 4;
    if (int e = go.check_error(s)) throw Error(e, "a net was left without a batch");
    batch_off.resize(nb + 1);
    class_off.resize(3 * (size_t)nb);
    for (int b = 0; b < nb; b++) {
        batch_off[b] = offs[3 * b];
        for (int c = 0; c < 3; c++) class_off[3 * b + c] = offs[3 * b + c];
    }
    batch_off[nb] = offs[3 * nb];
    if (batch_off[nb] != R) throw Error(ERR_STATE, "phase-1 plan does not cover every net");
}

// The per-batch launches of phase 1 (Lshape_route.hpp:235-242), stream-ordered.
void Router::emit_phase1(const std::vector<int> &batch_off, const std::vector<int> &class_off, bool timed) {
    const int nb = (int)batch_off.size() - 1;
    // the fused per-track commit holds tracks of up to kMaxFusedTrackCells cells
    const bool split = split || std::max(go.g.X, go.g.Y) > kMaxFusedTrackCells;
    cuda_check(cudaMemsetAsync(d_queue.p, 0, (3 * (size_t)nb + 1) * sizeof(int), s), "memset");
    for (int bi = 0; bi < nb; bi++) {
        const int off = batch_off[bi], n = batch_off[bi + 1] - off;
        const int stamp = bi + 1;
        if (seed_active && seed_levels > 0) {
            // the seed shrinks in `seed_levels` steps as the batches commit real demand
            const int lv = (int)((int64_t)bi * seed_levels / nb);
            if (bi == 0 || lv != (int)((int64_t)(bi - 1) * seed_levels / nb)) {
                launch_seed_step(go.g.N, go.demand.p, d_seed_dem.p, d_seed_cur.p, 1.f - (float)lv / seed_levels, s);
                go.mark_all_dirty(s);
                st.launches += 1;
            }
        }
        if (timed) kt.begin(split ? KC_COST : KC_COMMIT_REFRESH);
        if (split) launch_cost_refresh(go.g, true, s);
        else launch_commit_refresh(go.g, d_vcnt.p, bi, true, s);  // commits batch bi-1 (stamp bi)
        if (timed) kt.end(split ? KC_COST : KC_COMMIT_REFRESH);
        if (timed) kt.begin(KC_PATTERN);
        // batched form: the large (c = 0) and small (c = 2) classes are forked
        // onto their own streams and run beside the medium class (c = 1)
        bool forked[3] = {false, false, false};
        if (batched) cuda_check(cudaEventRecord(ev_fork, s), "event");
        for (int c = 0; c < 3; c++) {
            const int a = class_off[3 * bi + c];
            const int e = c < 2 ? class_off[3 * bi + c + 1] : batch_off[bi + 1];
            if (e <= a) continue;
            TreeBatchDev tb{d_ids.p + a, d_tree_off.p, d_tree_nodes.p, d_tree_par.p, d_route_off.p, d_route_cap.p,
                            routes.p, d_scratch.p, d_scratch_off.p, scratch_nodes, e - a};
            tb.queue = d_queue.p + 3 * bi + c;
            tb.vcnt = split ? nullptr : d_vcnt.p;
            cudaStream_t cs = s;
            if (batched) {
                tb.tile = c == 0 ? 32 : (c == 1 ? kPatternNodeTile : 6);
                tb.lanes_per_net = tune.lanes[c];
                if (c != 1) {
                    cs = s_cls[c == 0 ? 0 : 1];
                    cuda_check(cudaStreamWaitEvent(cs, ev_fork, 0), "fork");
                    forked[c] = true;
                }
            } else {
                tb.tile = kPatternNodeTile;  // nets beyond the tile use global scratch in the same launch
                tb.lanes_per_net = 32;  // 16 lanes: 3.16 -> 3.86 ms per c1 route
            }
            launch_pattern_route(go.g, tb, stamp, cs);
            st.launches += 1;
        }
        for (int c : {0, 2}) {
            if (!forked[c]) continue;
            const int j = c == 0 ? 0 : 1;
            cuda_check(cudaEventRecord(ev_join[j], s_cls[j]), "event");
            cuda_check(cudaStreamWaitEvent(s, ev_join[j], 0), "join");
        }
        if (timed) kt.end(KC_PATTERN);
        st.launches += 1;
        if (!split) continue;
        if (timed) kt.begin(KC_WIRE_COMMIT);
        launch_wire_commit(go.g, stamp, true, s);
        if (timed) kt.end(KC_WIRE_COMMIT);
        ViaBatchDev vb{d_ids.p + off, d_route_off.p, routes.p, n};
        if (timed) kt.begin(KC_VIA_COMMIT);
        launch_via_commit(go.g, vb, stamp, 1, s);
        if (timed) kt.end(KC_VIA_COMMIT);
        st.launches += 2;
    }
    if (!split && nb > 0) {  // commit of the last batch; its costs are refreshed when next needed
        if (timed) kt.begin(KC_COMMIT_REFRESH);
        launch_commit_refresh(go.g, d_vcnt.p, nb, false, s);
        if (timed) kt.end(KC_COMMIT_REFRESH);
        st.launches += 1;
    }
}

void Router::phase1() {
    const int R = (int)ns.nets.size();
    // colouring and plan stay on the device; only the batch and class offsets
    // come back to size the launches
    const int nb = run_color(R, d_perm1.p, d_shapes1, 15);
    st.batches1 = nb;
    if (batched && !tuned) autotune(nb);
    seed_begin();
    std::vector<int> batch_off, class_off;
    plan_phase1(nb, batch_off, class_off);
    grow_routes(route_end);
    cuda_check(cudaMemcpyAsync(d_route_off.p, d_route_off1.p, (size_t)R * 8, cudaMemcpyDeviceToDevice, s), "D2D");
    cuda_check(cudaMemcpyAsync(d_route_cap.p, d_route_cap1.p, (size_t)R * 4, cudaMemcpyDeviceToDevice, s), "D2D");
    d_queue.alloc(3 * (size_t)nb + 1);
    cuda_check(cudaEventRecord(ev0, s), "event");
    if (batched) {
        // the whole phase-1 loop as one CUDA graph, reused while the plan is unchanged
        const int gkey = seed_active ? 1 + seed_levels : 0;
        if (!graph1_exec || graph1_batch_off != batch_off || graph1_class_off != class_off || graph1_routes != routes.p ||
            graph1_seed != gkey) {
            if (graph1_exec) { cudaGraphExecDestroy(graph1_exec); graph1_exec = nullptr; }
            cudaGraph_t gr = nullptr;
            cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "capture");
            const long long l0 = st.launches;
            emit_phase1(batch_off, class_off, false);
            graph1_launches = st.launches - l0;
            cuda_check(cudaStreamEndCapture(s, &gr), "capture");
            cuda_check(cudaGraphInstantiate(&graph1_exec, gr, 0), "graph instantiate");
            cudaGraphDestroy(gr);
            graph1_batch_off = batch_off;
            graph1_class_off = class_off;
            graph1_routes = routes.p;
            graph1_seed = gkey;
        } else {
            st.launches += graph1_launches;
        }
        kt.begin(KC_GRAPH1);  // whole graph: cost refreshes, DP, commits
        cuda_check(cudaGraphLaunch(graph1_exec, s), "graph launch");
        kt.end(KC_GRAPH1);
    } else {
        emit_phase1(batch_off, class_off, true);
    }
    global_stamp = nb;
    cuda_check(cudaEventRecord(ev1, s), "event");
    cuda_check(cudaGetLastError(), "phase-1 launch");
    // plan of this run, in routing order (for igr_router_plan; ids fetched on demand)
    plan_batch_off.swap(batch_off);
    plan_ids.clear();
    plan_built = false;
    cuda_check(cudaEventSynchronize(ev1), "phase 1");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    st.p1_ms = ms;
    if (int e = go.check_error(s)) throw Error(e, "device error in phase 1");
    if (verbose) std::fprintf(stderr, "[igr] phase 1: %d batches, %.2f ms device\n", nb, ms);
}

// Autotuner of the batched form: picks the node count that separates small
// from medium nets and the lanes per net of each size class by timing the
// phase-1 batch loop of this design once per candidate (the routes are the
// same for every candidate).  Results are cached per grid and net count in
// $IGR_TUNE_CACHE (default ~/.cache/instantgr_b200/tune.txt).
static std::string tune_cache_path() {
    if (const char *p = std::getenv("IGR_TUNE_CACHE")) return p;
    const char *h = std::getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/instantgr_b200/tune.txt";
}

void Router::autotune(int nb) {
    const int R = (int)ns.nets.size();
    char key[96];
    std::snprintf(key, sizeof key, "%d %d %d %d", ns.X, ns.Y, R, nb);
    const std::string path = tune_cache_path();
    if (FILE *f = std::fopen(path.c_str(), "r")) {
        char line[256];
        while (std::fgets(line, sizeof line, f)) {
            int x, y, r, b, cl, sp, l0, l1, l2;
            if (std::sscanf(line, "%d %d %d %d %d %d %d %d %d", &x, &y, &r, &b, &cl, &sp, &l0, &l1, &l2) == 9) {
                char k2[96];
                std::snprintf(k2, sizeof k2, "%d %d %d %d", x, y, r, b);
                auto lanes_ok = [](int l) { return l == 16 || l == 32; };
                if (std::string(k2) == key && (cl == 1 || cl == 3) && sp >= 1 && sp <= 6 && lanes_ok(l0) &&
                    lanes_ok(l1) && lanes_ok(l2)) {
                    tune.classes = cl; tune.split = sp; tune.lanes[0] = l0; tune.lanes[1] = l1; tune.lanes[2] = l2;
                    tuned = true;
                }
            }
        }
        std::fclose(f);
        if (tuned) return;
    }
    std::vector<Tune> cands;
    for (int lm : {32, 16}) {
        Tune t;
        t.classes = 1; t.lanes[1] = lm;
        cands.push_back(t);
    }
    for (int sp : {3, 4, 6})
        for (int lm : {16, 32})
            for (int ls : {16, 32}) {
                Tune t;
                t.classes = 3; t.split = sp; t.lanes[0] = 32; t.lanes[1] = lm; t.lanes[2] = ls;
                cands.push_back(t);
            }
    Tune best = tune;
    float best_ms = 1e30f;
    std::vector<int> batch_off, class_off;
    d_queue.alloc(3 * (size_t)nb + 1);
    grow_routes(route_end);
    for (const Tune &cand : cands) {
            {
                tune = cand;
                plan_phase1(nb, batch_off, class_off);
                go.reset_demand(s);
                seed_begin();
                cuda_check(cudaMemcpyAsync(d_route_off.p, d_route_off1.p, (size_t)R * 8, cudaMemcpyDeviceToDevice, s), "D2D");
                cuda_check(cudaMemcpyAsync(d_route_cap.p, d_route_cap1.p, (size_t)R * 4, cudaMemcpyDeviceToDevice, s), "D2D");
                cuda_check(cudaEventRecord(ev0, s), "event");
                const long long l0 = st.launches;
                emit_phase1(batch_off, class_off, false);
                st.launches = l0;
                cuda_check(cudaEventRecord(ev1, s), "event");
                cuda_check(cudaEventSynchronize(ev1), "autotune");
                float ms = 0;
                cudaEventElapsedTime(&ms, ev0, ev1);
                if (ms < best_ms) { best_ms = ms; best = tune; }
            }
    }
    tune = best;
    tuned = true;
    go.reset_demand(s);
    if (go.check_error(s)) throw Error(ERR_STATE, "device error while autotuning");
    if (verbose)
        std::fprintf(stderr, "[igr] autotune: %d classes, split %d, lanes %d/%d/%d (%.2f ms)\n", tune.classes,
                     tune.split, tune.lanes[0], tune.lanes[1], tune.lanes[2], best_ms);
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        const std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); i++)
            if (i == dir.size() || dir[i] == '/') (void)mkdir(dir.substr(0, i).c_str(), 0755);
    }
    if (FILE *f = std::fopen(path.c_str(), "a")) {
        std::fprintf(f, "%s %d %d %d %d %d\n", key, tune.classes, tune.split, tune.lanes[0], tune.lanes[1],
                     tune.lanes[2]);
        std::fclose(f);
    }
}

// Trees and route capacities of the last phase-1 plan, in routing order.
void Router::build_plan() {
    if (plan_built) return;
    if (plan_ids.empty() && !plan_batch_off.empty()) {
        plan_ids.resize(plan_batch_off.back());
        cuda_check(cudaMemcpyAsync(plan_ids.data(), d_ids.p, plan_ids.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "plan");
    }
    plan_node_off.assign(1, 0);
    plan_nodes.clear();
    plan_par.clear();
    plan_cap.resize(plan_ids.size());
    for (size_t k = 0; k < plan_ids.size(); k++) {
        const int id = plan_ids[k];
        plan_nodes.insert(plan_nodes.end(), tree_nodes.begin() + tree_off[id], tree_nodes.begin() + tree_off[id + 1]);
        plan_par.insert(plan_par.end(), tree_par.begin() + tree_off[id], tree_par.begin() + tree_off[id + 1]);
        plan_node_off.push_back((int)plan_nodes.size());
        plan_cap[k] = route_cap1[id];
    }
    plan_built = true;
}

// Colours `order` (highest priority first) into batches of spatially disjoint
// nets (database_cuda.hpp:437-631); the colouring ranks the reversed list, so
// the first net of `order` wins every conflict.
void Router::color_nets(const std::vector<int> &order, const ShapeDev &shapes, int sparsity,
                        std::vector<std::vector<int>> &batches) {
    const int n = (int)order.size();
    batches.clear();
    if (n == 0) return;
    std::vector<int> perm(order.rbegin(), order.rend());
    d_perm.upload(perm, s);
    st.h2d_bytes += (int64_t)n * 4;
    const int nb = run_color(n, d_perm.p, shapes, sparsity);
    std::vector<int> bid(n);
    cuda_check(cudaMemcpyAsync(bid.data(), d_bat.p, n * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    st.d2h_bytes += (int64_t)n * 4;
    batches.assign(nb, {});
    for (int k = 0; k < n; k++) {
        if (bid[k] < 0 || bid[k] >= nb) throw Error(ERR_STATE, "a net was left without a batch");
        batches[bid[k]].push_back(perm[k]);
    }
}

int Router::run_color(int n, const int *d_perm_ranks, const ShapeDev &shapes, int sparsity) {
    d_map.alloc((size_t)ns.X * ns.Y);
    d_bat.alloc(n);
    d_act.alloc(4 * (size_t)n);
    d_hdr.alloc(n);
    d_flags.alloc(16);
    if (sparsity != shapes.sparsity) throw Error(ERR_STATE, "claim lists were built for another sparsity");
    ColorDev cd;
    cd.n = n; cd.X = ns.X; cd.Y = ns.Y; cd.sparsity = sparsity;
    cd.perm = d_perm_ranks;
    cd.pt_off = shapes.pt_off.p; cd.pts = shapes.pts.p; cd.pt_net = shapes.pt_net.p;
    cd.h_off = shapes.h_off.p; cd.hseg = shapes.hseg.p; cd.v_off = shapes.v_off.p; cd.vseg = shapes.vseg.p;
    cd.claim_off = shapes.claim_off.p; cd.claim = shapes.claim.p;
    cd.claim_n = shapes.claim_n.n ? shapes.claim_n.p : nullptr;
    cd.pt_n = shapes.pt_n.n ? shapes.pt_n.p : nullptr;
    cd.active = d_act.p; cd.active2 = d_act.p + n; cd.cand = d_act.p + 2 * (size_t)n; cd.lost = d_act.p + 3 * (size_t)n;
    cd.hdr = d_hdr.p;
    cd.ops = d_cops.p;
    cd.npts = shapes.npts; cd.map = d_map.p; cd.batch = d_bat.p; cd.flags = d_flags.p;
    // Round-0 map kept up to date across batches instead of re-claimed: it
    // pays on the largest colourings only (10M-net design: 1.57 s to 1.28 s
    // in phase 1, 12% in the rip-up passes), while the recomputation of the
    // cells whose owner joined costs about as much as the claims it saves on
    // designs of up to a million nets (130k-net design: 3.5 ms to 7.2 ms).
    if (n >= test_hooks().color_keep_min_nets.load() && shapes.claim.n < (size_t)INT32_MAX) {
        const size_t XY = (size_t)ns.X * ns.Y;
        d_rev_off.alloc(XY); d_rev_cnt.alloc(XY); d_rev.alloc(std::max<size_t>(1, shapes.claim.n));
        d_snap.alloc(XY); d_dirty.alloc(XY); d_part.alloc(1024);
        cd.rev_off = d_rev_off.p; cd.rev_cnt = d_rev_cnt.p; cd.rev = d_rev.p; cd.snap = d_snap.p;
        cd.dirty = d_dirty.p; cd.part = d_part.p;
    }
    const double t0 = verbose ? now_s() : 0;
    kt.begin(KC_COLOR);
    int nb = run_coloring(cd, 0, s);
    kt.end(KC_COLOR);
    if (verbose)
        std::fprintf(stderr, "[igr] colouring: %d nets, %zu claim cells, %d points, sparsity %d: %d batches, %d rounds, "
                     "%.2f ms\n", n, shapes.claim.n, shapes.npts, sparsity, nb, cd.rounds, (now_s() - t0) * 1e3);
    st.color_rounds += cd.rounds;
    st.launches += 1;
    if (nb == -2) throw Error(ERR_TIMEOUT, "colouring barrier timed out");
    if (nb < 0) throw Error(ERR_CUDA, std::string("colouring failed: ") + cudaGetErrorString(cudaGetLastError()));
    return nb;
}

// One rip-up-and-reroute pass (main.cpp:37-68, Lshape_route_detour.hpp:726-1112).
// Returns false when no net overflows.
// Positions into of_ids (ascending ids) in the order the pass reroutes them:
// decreasing HPWL, the reference's sort (Lshape_route_detour.hpp:732-734), or
// predicted congestion first with the seed's rip-up order.  Sorting the
// positions with the keys of their ids makes the comparisons and moves of
// sorting the ids themselves, hence the same order.
std::vector<int> Router::pass_order(const std::vector<int> &of_ids) const {
    const size_t K = of_ids.size();
    std::vector<int> ord(K);
    if (seed_active && seed_order) {
        std::vector<double> pr(K);
        for (size_t k = 0; k < K; k++) pr[k] = seed_pressure(of_ids[k]);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int l, int r) {
            if (pr[l] != pr[r]) return pr[l] > pr[r];
            return ns.nets[of_ids[l]].hpwl > ns.nets[of_ids[r]].hpwl;
        });
    } else {
        // (key, position) pairs compared on the key alone (the HPWL of every
        // routing net, kept since open)
        std::vector<std::pair<int, int>> kv(K);
        for (size_t k = 0; k < K; k++) kv[k] = {hpwl_keys[of_ids[k]], (int)k};
        std::sort(kv.begin(), kv.end(),
                  [](const std::pair<int, int> &l, const std::pair<int, int> &r) { return l.first > r.first; });
        for (size_t k = 0; k < K; k++) ord[k] = kv[k].second;
    }
    return ord;
}

bool Router::rrr_pass(int iter) {
    const int R = (int)ns.nets.size();
    const int X = ns.X, Y = ns.Y;
    if (R == 0) return false;
    const double tp0 = now_s();
    of_sum.alloc(go.g.N);
    d_is_of.alloc(R);
    d_xsum.alloc((size_t)X * Y);
    d_ysum.alloc((size_t)X * Y);
    // (the device's record offsets and capacities were brought up to date at
    // the end of the previous pass, or by phase 1)
    cuda_check(cudaEventRecord(ev0, s), "event");
    // overflow marking and congestion view (graph.hpp:588-601, main.cpp:42-45)
    ViaBatchDev all{d_all_ids.p, d_route_off.p, routes.p, R};
    kt.begin(KC_RIPUP);
    launch_mark_overflow(go.g, 0, of_sum.p, all, 10, d_is_of.p, s);
    kt.end(KC_RIPUP);
    // the flagged nets in id order, listed on the device
    d_of_list.alloc(R);
    d_of_blocks.alloc(std::max(1, flag_list_blocks(R)) + 1);
    launch_flag_list(d_is_of.p, R, d_of_list.p, d_of_blocks.p + flag_list_blocks(R), d_of_blocks.p, s);
    st.launches += 5;
    CongestionView cv;
    cv.X = X; cv.Y = Y;
    if (host_dags) {
        cv.xsum.resize((size_t)X * Y);
        cv.ysum.resize((size_t)X * Y);
    }
    int n_of = 0;
    cuda_check(cudaMemcpyAsync(&n_of, d_of_blocks.p + flag_list_blocks(R), sizeof(int), cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    std::vector<int> of_nets(n_of);
    if (n_of > 0) {
        cuda_check(cudaMemcpyAsync(of_nets.data(), d_of_list.p, (size_t)n_of * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "sync");
    }
    const double tp_mark = now_s();
    st.d2h_bytes += 4 + (int64_t)n_of * 4;
    st.rerouted = (int)of_nets.size();
    if (verbose) std::fprintf(stderr, "[igr] pass %d: %zu nets to reroute\n", iter, of_nets.size());
    if (of_nets.empty()) return false;
    // the host builds the detour DAGs from the congestion view (Lshape_route_detour.hpp:735-740)
    kt.begin(KC_RIPUP);
    launch_congestion_view(go.g, d_xsum.p, d_ysum.p, s);
    kt.end(KC_RIPUP);
    st.launches += 3;
    if (host_dags) {  // the host builder reads the view from host memory
        cuda_check(cudaMemcpyAsync(cv.xsum.data(), d_xsum.p, cv.xsum.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(cv.ysum.data(), d_ysum.p, cv.ysum.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "sync");
        st.d2h_bytes += (int64_t)X * Y * 8;
    }
    // per colour batch: its first entries in the arrays of the pass and its sizes
    std::vector<std::vector<int>> batches;
    std::vector<DagBatchInfo> bi;
    std::vector<int64_t> old_off;
    double th0 = now_s(), t_dag = 0, t_shapes = 0, t_color = 0, t_csr = 0;
    if (!host_dags) {
        // the pass order on a host thread while the device builds the DAGs in id order
        std::future<std::vector<int>> order =
            std::async(std::launch::async, [this, &of_nets] { return pass_order(of_nets); });
        double tm[4];
        if (!dags_on_device(of_nets, order, batches, bi, old_off, tm)) return false;
        t_dag = tm[0]; t_shapes = tm[1]; t_color = tm[2]; t_csr = tm[3];
    } else {
        {
            const std::vector<int> ord = pass_order(of_nets);
            std::vector<int> ids(ord.size());
            for (size_t k = 0; k < ord.size(); k++) ids[k] = of_nets[ord[k]];
            of_nets.swap(ids);
        }
        old_off = route_off;
        // detour DAGs on host threads (Lshape_route_detour.hpp:702-748)
        th0 = now_s();
        // DAGs of the rerouted nets only, by their position in of_nets; their arrays
        // come from one arena per range of nets, emptied at the next pass
        const int K = (int)of_nets.size();
        const int T = std::max(1, std::min(K, 8 * (threads > 0 ? threads : hw_threads())));
        auto task_begin = [&](int t) { return (int)((int64_t)K * t / T); };
        dag.clear();
        for (auto &a : dag_arenas) a->release();
        while ((int)dag_arenas.size() < T)
            dag_arenas.push_back(std::make_unique<std::pmr::monotonic_buffer_resource>(host_block_cache()));
        dag.reserve(K);
        for (int t = 0; t < T; t++)
            for (int k = task_begin(t); k < task_begin(t + 1); k++) dag.emplace_back(dag_arenas[t].get());
        dag_slot.assign(R, -1);
        for (size_t k = 0; k < of_nets.size(); k++) dag_slot[of_nets[k]] = (int)k;
        std::vector<char> keep(of_nets.size(), 1);
        parallel_for(T, threads, [&](int tb, int te) {
            for (int k = task_begin(tb); k < task_begin(te); k++) {
                DagNet &dn = dag[k];
                build_dag(ns, ns.nets[of_nets[k]], cv, mode_eff, dn);
                // the DP keeps at most 10 child slots per node (the reference packs the
                // slot as a decimal digit); nets beyond that keep their current route
                for (int c : dn.child_num)
                    if (c > 10) keep[k] = 0;
            }
        });
        {
            std::vector<int> kept;
            for (size_t k = 0; k < of_nets.size(); k++)
                if (keep[k]) kept.push_back(of_nets[k]);
            of_nets.swap(kept);
        }
        st.dag_host_ms += (now_s() - th0) * 1e3;
        t_dag = now_s();
        if (of_nets.empty()) return false;
        // colouring on DAG points and tree segments (Lshape_route_detour.hpp:751)
        // conflict shapes of the rerouted nets: their DAG points and their trees'
        // segments; claim lists built on the device
        std::vector<int> pt_off(of_nets.size() + 1, 0), pts;
        for (size_t k = 0; k < of_nets.size(); k++) pt_off[k + 1] = pt_off[k] + (int)dag[dag_slot[of_nets[k]]].points.size();
        pts.resize(pt_off.back());
        parallel_for((int)of_nets.size(), threads, [&](int b, int e) {
            for (int k = b; k < e; k++) {
                const auto &p = dag[dag_slot[of_nets[k]]].points;
                std::copy(p.begin(), p.end(), pts.begin() + pt_off[k]);
            }
        });
        d2_ptoff.upload(pt_off, s);
        d2_pts.upload(pts, s);
        d2_ids.upload(of_nets, s);
        st.h2d_bytes += (int64_t)(pt_off.size() + pts.size() + of_nets.size()) * 4;
        ShapeDev &shd = d_shapes2;
        {
            ShapeArgs a;
            a.tree_off = d_tree_off.p; a.tree_nodes = d_tree_nodes.p; a.tree_par = d_tree_par.p;
            a.ids = d2_ids.p; a.ext_off = d2_ptoff.p; a.ext_pts = d2_pts.p;
            a.n = (int)of_nets.size(); a.X = X; a.Y = Y; a.sparsity = mode_eff >= 1 ? 2 : 15;
            device_shapes(a, shd);
        }
        std::vector<int> local(of_nets.size());
        std::iota(local.begin(), local.end(), 0);  // shape k belongs to of_nets[k]; of_nets is in priority order
        std::vector<std::vector<int>> lb;
        t_shapes = now_s();
        color_nets(local, shd, mode_eff >= 1 ? 2 : 15, lb);
        t_color = now_s();
        batches.assign(lb.size(), {});
        for (size_t b = 0; b < lb.size(); b++)
            for (int k : lb[b]) batches[b].push_back(of_nets[k]);
        std::reverse(batches.begin(), batches.end());
        // batch-local CSR of all batches, laid end to end: sizes per net and batch
        // first, then every batch filled on its own thread
        const int B = (int)batches.size();
        bi.assign(B, DagBatchInfo{});
        std::vector<int> net_levels(of_nets.size()), net_slots(of_nets.size());  // depth + 1, child slots
        parallel_for((int)of_nets.size(), threads, [&](int b0, int e0) {
            for (int k = b0; k < e0; k++) {
                int D = 0, sl = 0;
                for (int dv : dag[k].depth) D = std::max(D, dv + 1);
                for (int c : dag[k].child_num) sl += c;
                net_levels[k] = D;
                net_slots[k] = sl;
            }
        });
        DagBatchInfo tot{};
        {
            DagBatchInfo acc{};
            for (int b = 0; b < B; b++) {
                DagBatchInfo &f = bi[b];
                f = acc;
                f.n = f.e = f.slots = f.mx_n = f.mx_e = 0;
                int lv = 0;
                for (int id : batches[b]) {
                    const int k = dag_slot[id];
                    const DagNet &dn = dag[k];
                    f.n += (int)dn.nodes.size();
                    f.e += (int)dn.par_nodes.size();
                    f.mx_n = std::max(f.mx_n, (int)dn.nodes.size());
                    f.mx_e = std::max(f.mx_e, (int)dn.par_nodes.size());
                    f.slots += net_slots[k];
                    lv += net_levels[k] + 1;
                    // new route record of the net (appended)
                    route_cap[id] = 8 * (int)dn.nodes.size() + 1;
                    route_off[id] = route_end;
                    route_end += route_cap[id];
                }
                if ((int64_t)f.n * 100 + 99 > 0x7fffffffLL) throw Error(ERR_CAPACITY, "DAG batch too large for 32-bit node ids");
                const int nn = (int)batches[b].size();
                const int64_t big = std::max({(int64_t)acc.pb + f.n + 1, (int64_t)acc.eb + f.e, (int64_t)acc.lb + lv,
                                              (int64_t)acc.nnb + nn + 1});
                if (big > 0x7fffffffLL) throw Error(ERR_CAPACITY, "DAG arrays of one rip-up pass exceed 32-bit offsets");
                acc.nb += f.n; acc.eb += f.e; acc.pb += f.n + 1; acc.lb += lv; acc.nnb += nn + 1; acc.nets += nn;
            }
            tot = acc;
        }
        // every entry is written below: left uninitialised (these reach billions of entries)
        HostArray<int> nodes(tot.nb), par_off(tot.pb), par(tot.eb), cslot(tot.eb), echild(tot.eb), child_off(tot.pb);
        HostArray<int> level_off(tot.lb), level_nodes(tot.nb), net_node_off(tot.nnb), net_ids(tot.nets),
            net_level_off(tot.nnb);
        parallel_for(B, threads, [&](int b0, int e0) {
            std::vector<int> dep, b_nodes, b_off, b_net;
            for (int b = b0; b < e0; b++) {
                const DagBatchInfo &f = bi[b];
                dep.resize(f.n);
                int e = 0, sl = 0, base = 0;
                par_off[f.pb] = 0;
                child_off[f.pb] = 0;
                net_node_off[f.nnb] = 0;
                int j = 0;
                for (int id : batches[b]) {
                    const DagNet &dn = dag[dag_slot[id]];
                    const int m = (int)dn.nodes.size();
                    for (int v = 0; v < m; v++) {
                        nodes[f.nb + base + v] = dn.nodes[v];
                        for (int q = dn.par_sum[v]; q < dn.par_sum[v + 1]; q++) {
                            par[f.eb + e] = base + dn.par_nodes[q];
                            cslot[f.eb + e] = dn.child_idx[q];
                            echild[f.eb + e] = base + v;
                            e++;
                        }
                        par_off[f.pb + base + v + 1] = e;
                        sl += dn.child_num[v];
                        child_off[f.pb + base + v + 1] = sl;
                        dep[base + v] = dn.depth[v];
                    }
                    base += m;
                    net_ids[f.nets + j] = id;
                    net_node_off[f.nnb + j + 1] = base;
                    j++;
                }
                // levels of each net of the batch (batch-local positions)
                dag_levels(j, net_node_off.data() + f.nnb, dep.data(), b_nodes, b_off, b_net);
                std::copy(b_nodes.begin(), b_nodes.end(), level_nodes.begin() + f.nb);
                std::copy(b_off.begin(), b_off.end(), level_off.begin() + f.lb);
                std::copy(b_net.begin(), b_net.end(), net_level_off.begin() + f.nnb);
            }
        });
        if (verbose) {
            // shape of the DAGs: nodes and depth per net, widest level of one net
            std::vector<int> nn, nd, nw;
            for (int id : of_nets) {
                const DagNet &dn = dag[dag_slot[id]];
                int dmax = 0;
                for (int dv : dn.depth) dmax = std::max(dmax, dv + 1);
                std::vector<int> w(dmax, 0);
                for (int dv : dn.depth) w[dv]++;
                nn.push_back((int)dn.nodes.size());
                nd.push_back(dmax);
                nw.push_back(dmax ? *std::max_element(w.begin(), w.end()) : 0);
            }
            for (auto *v : {&nn, &nd, &nw}) {  // counting sort: the values are small
                int mx = 0;
                for (int x : *v) mx = std::max(mx, x);
                std::vector<int64_t> h((size_t)mx + 2, 0);
                for (int x : *v) h[x]++;
                size_t k = 0;
                for (int x = 0; x <= mx; x++)
                    for (int64_t c = 0; c < h[x]; c++) (*v)[k++] = x;
            }
            auto q = [](const std::vector<int> &v, double p) {  // v sorted
                return v.empty() ? 0 : v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))];
            };
            std::fprintf(stderr,
                         "[igr] dags: %zu batches, %zu nets, %zu nodes; per net nodes p50 %d p90 %d p99 %d max %d, "
                         "depth p50 %d p90 %d p99 %d max %d, widest level p50 %d p99 %d max %d\n",
                         batches.size(), of_nets.size(), nodes.size(), q(nn, .5), q(nn, .9), q(nn, .99), q(nn, 1),
                         q(nd, .5), q(nd, .9), q(nd, .99), q(nd, 1), q(nw, .5), q(nw, .99), q(nw, 1));
        }
        t_csr = now_s();
        grow_routes(route_end);
        dg_nodes.upload(nodes.data(), nodes.size(), s); dg_paroff.upload(par_off.data(), par_off.size(), s);
        dg_par.upload(par.data(), par.size(), s); dg_cslot.upload(cslot.data(), cslot.size(), s);
        dg_echild.upload(echild.data(), echild.size(), s); dg_childoff.upload(child_off.data(), child_off.size(), s);
        dg_leveloff.upload(level_off.data(), level_off.size(), s);
        dg_levelnodes.upload(level_nodes.data(), level_nodes.size(), s);
        dg_nno.upload(net_node_off.data(), net_node_off.size(), s); dg_ids.upload(net_ids.data(), net_ids.size(), s);
        dg_netlvl.upload(net_level_off.data(), net_level_off.size(), s);
        d_old_off.upload(old_off, s);
        d_route_off.upload(route_off, s);
        d_route_cap.upload(route_cap, s);
        st.h2d_bytes += (int64_t)(nodes.size() * 2 + par_off.size() * 2 + par.size() * 3 + level_off.size() +
                                  net_level_off.size() + net_node_off.size() + net_ids.size()) * 4 + (int64_t)R * 20;
    }
    int mn = 1, me = 1, ms = 1;
    for (auto &f : bi) { mn = std::max(mn, f.n); me = std::max(me, f.e); ms = std::max(ms, f.slots); }
    dg_costs.alloc((size_t)mn * 10); dg_cedges.alloc((size_t)me * 81); dg_offers.alloc((size_t)me * 54);
    dg_best.alloc((size_t)ms * 10); dg_packed.alloc((size_t)ms * 10);
    dg_bchange.alloc((size_t)me * 81); dg_lout.alloc(mn); dg_stage.alloc((size_t)mn * 8); dg_scnt.alloc(mn);
    for (size_t b = 0; b < bi.size(); b++) {
        const DagBatchInfo &f = bi[b];
        const int nnet = (int)batches[b].size();
        if (b == 1 && gather_pending) {  // the later batches' DAGs were gathered on a side stream
            cuda_check(cudaStreamWaitEvent(s, ev_gjoin, 0), "join");
            gather_pending = false;
        }
        ViaBatchDev old{dg_ids.p + f.nets, d_old_off.p, routes.p, nnet};
        const int s1 = ++global_stamp;
        kt.begin(KC_RIPUP);
        launch_wire_ripup(go.g, old, s1, -1, s);
        launch_via_commit(go.g, old, s1, -1, s);
        kt.end(KC_RIPUP);
        const int s2 = ++global_stamp;
        kt.begin(KC_COST);
        launch_cost_refresh(go.g, true, s);
        kt.end(KC_COST);
        DagBatchDev db;
        db.n_nodes = f.n; db.n_edges = f.e; db.n_nets = nnet;
        db.nodes = dg_nodes.p + f.nb; db.par_off = dg_paroff.p + f.pb; db.par = dg_par.p + f.eb;
        db.child_slot = dg_cslot.p + f.eb; db.edge_child = dg_echild.p + f.eb; db.child_off = dg_childoff.p + f.pb;
        db.level_off = dg_leveloff.p + f.lb; db.level_nodes = dg_levelnodes.p + f.nb;
        db.net_level_off = dg_netlvl.p + f.nnb;
        db.net_node_off = dg_nno.p + f.nnb; db.net_ids = dg_ids.p + f.nets;
        db.costs = dg_costs.p; db.best_path = dg_best.p; db.packed = dg_packed.p; db.cost_edges = dg_cedges.p;
        db.best_change = dg_bchange.p; db.layer_out = dg_lout.p; db.stage = dg_stage.p; db.stage_cnt = dg_scnt.p;
        db.route_off = d_route_off.p; db.route_cap = d_route_cap.p; db.routes = routes.p;
        kt.begin(KC_DAG);
        db.max_net_nodes = f.mx_n; db.max_net_edges = f.mx_e; db.offers = dg_offers.p;
        const int nl = launch_dag_route(go.g, db, s2, s, s_cls[0], ev_fork, ev_join[0],
                                        test_hooks().dag_split_nets.load(), test_hooks().dag_stage_nodes.load());
        kt.end(KC_DAG);
        kt.begin(KC_WIRE_COMMIT);
        launch_wire_commit(go.g, s2, true, s);
        kt.end(KC_WIRE_COMMIT);
        ViaBatchDev nw{dg_ids.p + f.nets, d_route_off.p, routes.p, nnet};
        kt.begin(KC_VIA_COMMIT);
        launch_via_commit(go.g, nw, s2, 1, s);
        kt.end(KC_VIA_COMMIT);
        st.launches += 5 + nl;
    }
    const double t_enq = now_s();  // every batch of the pass enqueued
    cuda_check(cudaEventRecord(ev1, s), "event");
    cuda_check(cudaGetLastError(), "reroute launch");
    cuda_check(cudaEventSynchronize(ev1), "reroute");
    dt_pack.release();  // the trees' copies are done
    float ms_ = 0;
    cudaEventElapsedTime(&ms_, ev0, ev1);
    st.rrr_ms += ms_;
    if (int e = go.check_error(s)) throw Error(e, "device error in rip-up and reroute");
    if (verbose)
        std::fprintf(stderr,
                     "[igr] pass %d host: marking and order %.3f s (marking on the device %.3f s), DAGs %.3f s, conflict "
                     "shapes %.3f s, colouring %.3f s, batch arrays %.3f s, batches on the device %.3f s (of it enqueueing "
                     "%zu batches %.3f s)\n",
                     iter, th0 - tp0, tp_mark - tp0, t_dag - th0, t_shapes - t_dag, t_color - t_shapes, t_csr - t_color,
                     now_s() - t_csr, bi.size(), t_enq - t_csr);
    return true;
}

void Router::PackedTrees::release() {
    pinned_free(off, n_off * sizeof(int));
    pinned_free(pos, n_pos * sizeof(int));
    pinned_free(aoff, n_aoff * sizeof(int));
    pinned_free(adj, n_adj * sizeof(int));
    off = pos = aoff = adj = nullptr;
    n_off = n_pos = n_aoff = n_adj = 0;
}

void Router::pack_dag_trees() {
    const int R = (int)ns.nets.size();
    std::vector<int64_t> off((size_t)R + 1, 0), aoff((size_t)R + 1, 0);
    parallel_for(R, threads, [&](int b, int e) {
        for (int r = b; r < e; r++) {
            off[r + 1] = (int64_t)ns.nets[r].tnode.size();
            aoff[r + 1] = (int64_t)ns.nets[r].adj.nb.size();
        }
    });
    for (int r = 0; r < R; r++) {
        off[r + 1] += off[r];
        aoff[r + 1] += aoff[r];
    }
    if (off[R] + 1 > INT32_MAX || aoff[R] > INT32_MAX) throw Error(ERR_CAPACITY, "trees exceed 32-bit offsets");
    // written in full below, by the threads that fill them
    const size_t nt = (size_t)off[R], na = (size_t)aoff[R];
    PackedTrees &p = dt_pack;
    p.release();
    p.n_off = (size_t)R + 1; p.n_pos = std::max<size_t>(nt, 1); p.n_aoff = nt + 1; p.n_adj = std::max<size_t>(na, 1);
    p.off = static_cast<int *>(pinned_alloc(p.n_off * sizeof(int)));
    p.pos = static_cast<int *>(pinned_alloc(p.n_pos * sizeof(int)));
    p.aoff = static_cast<int *>(pinned_alloc(p.n_aoff * sizeof(int)));
    p.adj = static_cast<int *>(pinned_alloc(p.n_adj * sizeof(int)));
    parallel_for(R, threads, [&](int b, int e) {
        for (int r = b; r < e; r++) {
            const RNet &n = ns.nets[r];
            const int base = (int)off[r], nbase = (int)aoff[r], T = (int)n.tnode.size();
            p.off[r] = base;
            for (int i = 0; i < T; i++) {
                p.pos[base + i] = n.tnode[i];
                p.aoff[base + i] = nbase + n.adj.off[i];
            }
            std::copy(n.adj.nb.begin(), n.adj.nb.end(), p.adj + nbase);
        }
    });
    p.off[R] = (int)nt;
    p.aoff[nt] = (int)na;
}

void Router::upload_dag_trees() {
    if (dt_ready) return;
    if (dt_packing.valid()) dt_packing.get();  // packed beside phase 1 (rethrows its error)
    else pack_dag_trees();
    const PackedTrees &p = dt_pack;
    const size_t nt = p.n_aoff - 1;
    // stream-ordered copies from page-locked memory; the buffers are given back
    // once the pass has synchronised
    d_dt_off.upload(p.off, p.n_off, s);
    d_dt_pos.upload(p.pos, nt, s);
    d_dt_aoff.upload(p.aoff, p.n_aoff, s);
    d_dt_adj.upload(p.adj, (size_t)p.aoff[nt], s);
    st.h2d_bytes += (int64_t)(p.n_off + 2 * nt + 1 + (size_t)p.aoff[nt]) * 4;
    dt_ready = true;
}

// Detour DAGs of the rerouted nets built on the device (dagbuild.cu), their
// conflict shapes and colouring, and the batch-local arrays of every colour
// batch gathered on the device: the batches and arrays of the host path.
// of_nets: the nets to reroute in id order on entry (DAG k is built for
// of_nets[k]), the ones rerouted in pass order (`order`, positions into the
// entry list, computed meanwhile) on return.
bool Router::dags_on_device(std::vector<int> &of_nets, std::future<std::vector<int>> &order,
                            std::vector<std::vector<int>> &batches, std::vector<DagBatchInfo> &bi,
                            const std::vector<int64_t> &, double *tm) {
    const int X = ns.X, Y = ns.Y, R = (int)ns.nets.size();
    const double th0 = now_s();
    upload_dag_trees();
    DagBuildArgs a;
    a.tree_off = d_dt_off.p; a.pos = d_dt_pos.p; a.adj_off = d_dt_aoff.p; a.adj = d_dt_adj.p;
    a.xsum = d_xsum.p; a.ysum = d_ysum.p; a.X = X; a.Y = Y; a.mode = mode_eff;
    d2_ids.upload(of_nets, s);
    st.h2d_bytes += (int64_t)of_nets.size() * 4;
    a.ids = d2_ids.p;
    a.n_list = (int)of_nets.size();
    // build order: tree nodes, then HPWL (nets alike in size side by side)
    std::vector<int> okey(of_nets.size());
    for (size_t k = 0; k < of_nets.size(); k++) {
        const RNet &rn = ns.nets[of_nets[k]];
        okey[k] = (int)std::min<size_t>(rn.tnode.size(), 32767) * 65536 + std::min(65535, rn.hpwl);
    }
    const double tb0 = now_s();
    ddag.build(a, s, &okey);
    const double tb1 = now_s();
    st.d2h_bytes += (int64_t)of_nets.size() * kDagSizeFields * 4;
    // in pass order, the DAGs of the nets rerouted: the DP keeps at most 10
    // child slots per node (the reference packs the slot as a decimal digit);
    // nets beyond that keep their current route
    const std::vector<int> ord = order.get();
    std::vector<int> kept;
    kept.reserve(of_nets.size());
    for (int k : ord)
        if (ddag.sz(k, 5) <= 10) kept.push_back(k);
    bool in_place = kept.size() == of_nets.size();  // kept[i] == i
    for (size_t i = 0; in_place && i < kept.size(); i++) in_place = kept[i] == (int)i;
    {
        std::vector<int> ids(kept.size());
        for (size_t i = 0; i < kept.size(); i++) ids[i] = of_nets[kept[i]];
        of_nets.swap(ids);
    }
    if (of_nets.empty()) return false;
    const int n = (int)of_nets.size();
    st.dag_host_ms += (now_s() - th0) * 1e3;
    tm[0] = now_s();
    // conflict shapes of the rerouted nets: their DAG points and their trees'
    // segments (Lshape_route_detour.hpp:751)
    ShapeDev &shd = d_shapes2;
    {
        ShapeArgs sa;
        sa.tree_off = d_tree_off.p; sa.tree_nodes = d_tree_nodes.p; sa.tree_par = d_tree_par.p;
        sa.ext_pts = ddag.points.p;
        if (in_place) {  // shape i is DAG i
            sa.ids = d2_ids.p;
            sa.ext_at = ddag.point_at.p; sa.ext_cnt = ddag.sizes.p + 2; sa.ext_stride = kDagSizeFields;
        } else {         // shape i is DAG kept[i]
            const double tk0 = now_s();
            std::vector<int> cnt(n);
            for (int i = 0; i < n; i++) cnt[i] = ddag.sz(kept[i], 2);
            d_kept.upload(of_nets, s);
            d_kept_dag.upload(kept, s);
            d2_extat.alloc(n);
            launch_take_i64(n, d_kept_dag.p, ddag.point_at.p, d2_extat.p, s);
            d2_ptoff.upload(cnt, s);
            st.launches += 1;
            sa.ids = d_kept.p; sa.ext_at = d2_extat.p; sa.ext_cnt = d2_ptoff.p; sa.ext_stride = 1;
            if (verbose) std::fprintf(stderr, "[igr] shape sources of %d nets: %.4f s\n", n, now_s() - tk0);
        }
        sa.n = n; sa.X = X; sa.Y = Y; sa.sparsity = mode_eff >= 1 ? 2 : 15;
        device_shapes(sa, shd);
    }
    tm[1] = now_s();
    std::vector<int> local(n);
    std::iota(local.begin(), local.end(), 0);  // shape i belongs to of_nets[i]; of_nets is in priority order
    std::vector<std::vector<int>> lb;
    color_nets(local, shd, mode_eff >= 1 ? 2 : 15, lb);
    tm[2] = now_s();
    // batches in the host path's order (last colour first), as ids and as positions
    const int B = (int)lb.size();
    batches.assign(B, {});
    std::vector<std::vector<int>> bpos(B);
    for (int b = 0; b < B; b++) {
        bpos[B - 1 - b] = lb[b];
        for (int i : lb[b]) batches[B - 1 - b].push_back(of_nets[i]);
    }
    auto m_of = [&](int i) { return ddag.sz(kept[i], 0); };
    auto e_of = [&](int i) { return ddag.sz(kept[i], 1); };
    auto d_of = [&](int i) { return ddag.sz(kept[i], 3); };
    auto s_of = [&](int i) { return ddag.sz(kept[i], 4); };
    // within a batch the largest DAGs first: the DP's CTAs start in that order,
    // so that the longest nets do not begin last (the nets of a batch are
    // independent; c2: 219 -> 215 ms per route)
    parallel_for(B, threads, [&](int b0, int e0) {
        for (int b = b0; b < e0; b++) {
            std::vector<int> &v = bpos[b];
            std::stable_sort(v.begin(), v.end(), [&](int l, int r) { return m_of(l) > m_of(r); });
            batches[b].clear();
            for (int i : v) batches[b].push_back(of_nets[i]);
        }
    });
    bi.assign(B, DagBatchInfo{});
    DagBatchInfo tot{};
    {
        DagBatchInfo acc{};
        for (int b = 0; b < B; b++) {
            DagBatchInfo &f = bi[b];
            f = acc;
            f.n = f.e = f.slots = f.mx_n = f.mx_e = 0;
            int64_t lv = 0;
            for (int i : bpos[b]) {
                const int id = of_nets[i];
                f.n += m_of(i);
                f.e += e_of(i);
                f.mx_n = std::max(f.mx_n, m_of(i));
                f.mx_e = std::max(f.mx_e, e_of(i));
                f.slots += s_of(i);
                lv += d_of(i) + 1;
                // new route record of the net (appended)
                route_cap[id] = 8 * m_of(i) + 1;
                route_off[id] = route_end;
                route_end += route_cap[id];
            }
            if ((int64_t)f.n * 100 + 99 > 0x7fffffffLL) throw Error(ERR_CAPACITY, "DAG batch too large for 32-bit node ids");
            const int nn = (int)bpos[b].size();
            const int64_t big = std::max({(int64_t)acc.pb + f.n + 1, (int64_t)acc.eb + f.e, (int64_t)acc.lb + lv,
                                          (int64_t)acc.nnb + nn + 1});
            if (big > 0x7fffffffLL) throw Error(ERR_CAPACITY, "DAG arrays of one rip-up pass exceed 32-bit offsets");
            acc.nb += f.n; acc.eb += f.e; acc.pb += f.n + 1; acc.lb += (int)lv; acc.nnb += nn + 1; acc.nets += nn;
        }
        tot = acc;
    }
    // gather layout: per net (batch order) its DAG and its bases in the batch
    std::vector<int> desc((size_t)n * kDagDescFields), bat((size_t)std::max(B, 1) * kDagBatchFields);
    parallel_for(B, threads, [&](int b0, int e0) {
        for (int b = b0; b < e0; b++) {
            const DagBatchInfo &f = bi[b];
            int base = 0, ebl = 0, sl = 0, lvb = 0, jl = 0;
            for (int i : bpos[b]) {
                int *d = desc.data() + (size_t)(f.nets + jl) * kDagDescFields;
                d[0] = kept[i]; d[1] = base; d[2] = ebl; d[3] = sl; d[4] = lvb; d[5] = jl; d[6] = b;
                base += m_of(i); ebl += e_of(i); sl += s_of(i); lvb += d_of(i) + 1; jl++;
            }
            int *t = bat.data() + (size_t)b * kDagBatchFields;
            t[0] = f.nb; t[1] = f.eb; t[2] = f.pb; t[3] = f.lb; t[4] = f.nnb; t[5] = f.nets;
        }
    });
    d_gdesc.upload(desc, s);
    d_gbatch.upload(bat, s);
    st.h2d_bytes += (int64_t)(desc.size() + bat.size()) * 4;
    dg_nodes.alloc(std::max(1, tot.nb)); dg_paroff.alloc(std::max(1, tot.pb)); dg_par.alloc(std::max(1, tot.eb));
    dg_cslot.alloc(std::max(1, tot.eb)); dg_echild.alloc(std::max(1, tot.eb)); dg_childoff.alloc(std::max(1, tot.pb));
    dg_leveloff.alloc(std::max(1, tot.lb)); dg_levelnodes.alloc(std::max(1, tot.nb));
    dg_nno.alloc(std::max(1, tot.nnb)); dg_ids.alloc(std::max(1, tot.nets)); dg_netlvl.alloc(std::max(1, tot.nnb));
    DagGatherArgs g;
    g.n = n; g.desc = d_gdesc.p; g.batch = d_gbatch.p; g.ids = d2_ids.p; g.sizes = ddag.sizes.p;
    g.node_at = ddag.node_at.p; g.edge_at = ddag.edge_at.p;
    g.src_nodes = ddag.nodes.p; g.src_par_num = ddag.par_num.p; g.src_child_num = ddag.child_num.p;
    g.src_depth = ddag.depth.p; g.src_par = ddag.par.p; g.src_child_idx = ddag.child_idx.p;
    g.nodes = dg_nodes.p; g.par_off = dg_paroff.p; g.par = dg_par.p; g.child_slot = dg_cslot.p;
    g.edge_child = dg_echild.p; g.child_off = dg_childoff.p; g.level_off = dg_leveloff.p;
    g.level_nodes = dg_levelnodes.p; g.net_node_off = dg_nno.p; g.net_ids = dg_ids.p; g.net_level_off = dg_netlvl.p;
    // the first batch's DAGs on the router's stream, the later batches' on a
    // side stream beside the first batch's kernels (batch 1 waits for them)
    const int n_first = B > 1 ? bi[1].nets : n;
    if (n_first < n) {
        cuda_check(cudaEventRecord(ev_gfork, s), "event");
        cuda_check(cudaStreamWaitEvent(s_cls[1], ev_gfork, 0), "fork");
    }
    DagGatherArgs g0 = g;
    g0.n = n_first;
    launch_dag_gather(g0, s);
    st.launches += 1;
    if (n_first < n) {
        DagGatherArgs g1 = g;
        g1.desc = g.desc + (size_t)n_first * kDagDescFields;
        g1.n = n - n_first;
        launch_dag_gather(g1, s_cls[1]);
        cuda_check(cudaEventRecord(ev_gjoin, s_cls[1]), "event");
        gather_pending = true;
        st.launches += 1;
    }
    cuda_check(cudaGetLastError(), "DAG gather launch");
    if (verbose) {
        int64_t mx = 0, dmx = 0, tn = 0, te = 0, tp = 0;
        for (int i = 0; i < n; i++) {
            mx = std::max<int64_t>(mx, m_of(i));
            dmx = std::max<int64_t>(dmx, d_of(i));
            tn += m_of(i); te += e_of(i); tp += ddag.sz(kept[i], 2);
        }
        int cls[3] = {0, 0, 0};
        for (int k : kept) cls[ddag.tier[k]]++;
        std::fprintf(stderr,
                     "[igr] dags on the device: %d batches, %d nets, %lld nodes, %lld edges, %lld points; max %lld nodes, "
                     "depth %lld; work-area classes %d/%d/%d; trees %.3f s, build %.3f s\n",
                     B, n, (long long)tn, (long long)te, (long long)tp, (long long)mx, (long long)dmx, cls[0], cls[1],
                     cls[2], tb0 - th0, tb1 - tb0);
    }
    tm[3] = now_s();
    grow_routes(route_end);
    // the offsets before this pass's records (the device's are still those),
    // then the new record slots of the rerouted nets
    d_old_off.alloc(R);
    cuda_check(cudaMemcpyAsync(d_old_off.p, d_route_off.p, (size_t)R * 8, cudaMemcpyDeviceToDevice, s), "D2D");
    {
        std::vector<int64_t> slot((size_t)3 * n);
        for (int i = 0; i < n; i++) {
            const int id = of_nets[i];
            slot[3 * i] = id;
            slot[3 * i + 1] = route_off[id];
            slot[3 * i + 2] = route_cap[id];
        }
        d_slots.upload(slot, s);
        launch_record_slots(n, d_slots.p, d_route_off.p, d_route_cap.p, s);
        st.h2d_bytes += (int64_t)n * 24;
        st.launches += 1;
    }
    return true;
}

void Router::compute_score() {
    unsigned long long h[kStatSlots] = {0, 0, 0, 0, 0};
    double of = 0;
    launch_overflow_cost(go.g, go.score.p, s);
    st.launches += 2;
    unsigned long long cops[5] = {0, 0, 0, 0, 0};
    if (d_cops.p) cuda_check(cudaMemcpyAsync(cops, d_cops.p, sizeof cops, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(h, go.stats.p, sizeof h, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(&of, go.score.p, sizeof of, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (pin_vias < 0) {
        pin_vias = 0;
        for (size_t i = 0; i < d.sel.size(); i++) pin_vias += d.sel[i] < d.X * d.Y;
    }
    // per claimed cell: 4-byte index + 8-byte read-modify-write; per point check:
    // index + owner (+ batch of the owner when blocking); per release check:
    // index + owner; per list entry scanned: entry + batch
    color_bytes = 12.0 * cops[0] + 8.0 * cops[1] + 12.0 * cops[2] + 8.0 * cops[3] + 8.0 * cops[4];
    cost_cells = h[2];
    commit_cells = h[3];
    commit_refresh_cells = h[4];
    score_wl = (double)(int64_t)h[0] * d.unit_wire;
    score_via = (double)((int64_t)h[1] + pin_vias) * d.unit_via;
    score_of = of;
}

void Router::evaluate(double *out, double *layer_loss) {
    if (!ran) throw Error(ERR_STATE, "route before evaluating");
    const int N = d.num_nets(), L = go.g.L, X = d.X, Y = d.Y;
    const int64_t XY = (int64_t)X * Y;
    EvalDev e;
    e.n = N; e.L = L; e.X = X; e.Y = Y; e.DIR = go.g.DIR;
    ev_sel_off.upload(d.sel_off, s); ev_sel.upload(d.sel, s);
    ev_extra_off.upload(d.extra_off, s); ev_extra.upload(d.extra, s);
    ev_sub_off.upload(ns.sub_off, s);
    ev_route_off.upload(route_off, s);
    e.sel_off = ev_sel_off.p; e.sel = ev_sel.p; e.extra_off = ev_extra_off.p; e.extra = ev_extra.p;
    e.sub_off = ev_sub_off.p; e.route_off = ev_route_off.p; e.routes = routes.p;
    e.cap = go.g.cap; e.xlen = go.g.xlen; e.ylen = go.g.ylen; e.err = go.g.err;
    if (!d.cap_d.empty()) {  // capacities that are not floats: the exact values, in the track layout
        ev_capd_ref.upload(d.cap_d.data() + XY, (size_t)L * XY, s);
        ev_capd.alloc((size_t)L * XY);
        launch_to_track_layout_d(go.g, ev_capd_ref.p, ev_capd.p, s);
        e.cap_d = ev_capd.p;
    }
    ev_wire.alloc((size_t)go.g.N);
    ev_stacked.alloc((size_t)go.g.N);
    cuda_check(cudaMemsetAsync(ev_wire.p, 0, (size_t)go.g.N * sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(ev_stacked.p, 0, (size_t)go.g.N * sizeof(int), s), "memset");
    ev_cnt.alloc(kEvalLayers + L);
    cuda_check(cudaMemsetAsync(ev_cnt.p, 0, (kEvalLayers + L) * sizeof(unsigned long long), s), "memset");
    e.wire = ev_wire.p; e.stacked = ev_stacked.p; e.total_vias = ev_cnt.p; e.wl = ev_cnt.p + kEvalLayers;
    // counts per design net, then the via-location offsets and the table sizes
    ev_vcnt.alloc(std::max(N, 1)); ev_ccnt.alloc(std::max(N, 1));
    launch_eval_count(e, ev_vcnt.p, ev_ccnt.p, s);
    std::vector<long long> vc(N), cc(N);
    if (N) {
        cuda_check(cudaMemcpyAsync(vc.data(), ev_vcnt.p, N * sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(cc.data(), ev_ccnt.p, N * sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
    }
    cuda_check(cudaStreamSynchronize(s), "evaluation counts");
    std::vector<long long> voff(N + 1, 0);
    long long ncell = 0;
    for (int i = 0; i < N; i++) { voff[i + 1] = voff[i] + vc[i]; ncell += cc[i]; }
    const long long nloc = voff[N];
    if (N > (1 << 28) || X > 65535 || Y > 65535) throw Error(ERR_CAPACITY, "design too large for the evaluation keys");
    auto table = [](long long n) {
        unsigned long long t = 64;
        while (t < 2ull * (unsigned long long)n) t <<= 1;
        return t;
    };
    const unsigned long long wt = table(ncell), vt = table(nloc);
    ev_voff.upload(voff.data(), N + 1, s);
    ev_wkeys.alloc(wt); ev_vkeys.alloc(vt); ev_vfirst.alloc(vt);
    ev_vloc.alloc(std::max<long long>(nloc, 1)); ev_vord.alloc(std::max<long long>(nloc, 1));
    cuda_check(cudaMemsetAsync(ev_wkeys.p, 0xff, wt * 8, s), "memset");
    cuda_check(cudaMemsetAsync(ev_vkeys.p, 0xff, vt * 8, s), "memset");
    cuda_check(cudaMemsetAsync(ev_vfirst.p, 0xff, vt * 4, s), "memset");
    e.wkeys = ev_wkeys.p; e.wmask = wt - 1; e.vkeys = ev_vkeys.p; e.vmask = vt - 1;
    e.vfirst = ev_vfirst.p; e.vloc = ev_vloc.p; e.vord = ev_vord.p;
    launch_eval_marks(e, ev_voff.p, nloc, s);
    const int bpl = eval_blocks_per_layer(XY);
    ev_part.alloc((size_t)bpl * L);
    launch_eval_cells(e, bpl, ev_part.p, s);
    std::vector<double> part((size_t)bpl * L);
    std::vector<unsigned long long> cnt(kEvalLayers + L);
    cuda_check(cudaMemcpyAsync(part.data(), ev_part.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(cnt.data(), ev_cnt.p, cnt.size() * 8, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "evaluation");
    cuda_check(cudaGetLastError(), "evaluation launch");
    if (int err = go.check_error(s)) throw Error(err, "device error in the evaluation");
    // per file layer in the evaluator's order: layer 0 is not a routing layer
    double wl_cost = 0, via_cost = 0, of_cost = 0;
    via_cost += double(cnt[0]) * d.unit_via;
    for (int z = 1; z <= L; z++) {
        double layer = 0;
        for (int b = 0; b < bpl; b++) layer += part[(size_t)(z - 1) * bpl + b];
        if (layer_loss) layer_loss[z - 1] = layer;
        of_cost += layer * d.short_cost[z];
        via_cost += double(cnt[z < kEvalLayers ? z : kEvalLayers - 1]) * d.unit_via;
        wl_cost += double(cnt[kEvalLayers + z - 1]) * d.unit_wire;
    }
    out[0] = wl_cost;
    out[1] = via_cost;
    out[2] = of_cost;
    out[3] = of_cost + via_cost + wl_cost;
}

void Router::write(const char *out) {
    const double t0 = now_s();
    fetch_routes();
    const double t1 = now_s();
    RouteSource rs;
    rs.routes_of = [&](int net) -> const int * { return route_end == 0 ? nullptr : route_of(net); };
    write_guides(d, ns, rs, out, threads);
    if (verbose) std::fprintf(stderr, "[igr] routes to host %.3fs, guides written %.3fs\n", t1 - t0, now_s() - t1);
}

}  // namespace igr
