// Host driver of the router and ownership of device memory.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <exception>
#include <future>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "device.hpp"
#include "host.hpp"

namespace igr {

void cuda_check(cudaError_t e, const char *what);
bool cuda_driver_ready();

// Process-wide cache of device memory: blocks given back stay mapped and are
// handed out again for requests of up to their size (per device), so that
// routers opened one after another do not pay cudaMalloc/cudaFree each time.
// A block is cached only after a device synchronisation, as cudaFree would.
void *dev_alloc(size_t bytes);
void dev_free(void *p, size_t bytes);
// cudaMalloc calls of the device cache so far, their total time (us) and cache trims
void dev_alloc_stats(long long *mallocs, long long *us, long long *trims);
// returns every cached block of the current device to the driver
void dev_trim();
// The same for page-locked host memory (cudaMallocHost), used for the copies
// of results to the host.
void *pinned_alloc(size_t bytes);
void pinned_free(void *p, size_t bytes);
// true when the cache holds a page-locked block for `bytes`
bool pinned_cached(size_t bytes);

template <typename T>
struct PinnedBuf {
    T *p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() { release(); }
    void release() {
        if (p) pinned_free(p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    // grow-only
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) count = 1;
        p = static_cast<T *>(pinned_alloc(count * sizeof(T)));
        n = count;
    }
};

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) dev_free(p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    // grow-only: reuses the allocation when it is large enough
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) count = 1;
        p = static_cast<T *>(dev_alloc(count * sizeof(T)));
        n = count;
    }
    void upload(const T *h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) cuda_check(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
    }
    void upload(const std::vector<T> &v, cudaStream_t s) { upload(v.data(), v.size(), s); }
};

// Colour batch of a rip-up pass: its first entries in the pass-wide DAG
// arrays (nodes, edges, nodes + 1 per net, depth levels, nets + 1, nets) and
// its node, edge and child-slot counts.
// Allocator whose value construction leaves ints uninitialised, for host
// arrays that are filled in parallel right after they are sized (a serial zero
// fill of the trees of 1.39M routing nets costs tens of milliseconds).
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) {}
    template <class U, class... A>
    void construct(U *p, A &&...a) {
        if constexpr (sizeof...(A) == 0) ::new ((void *)p) U;
        else ::new ((void *)p) U(std::forward<A>(a)...);
    }
};

struct DagBatchInfo {
    int nb, eb, pb, lb, nnb, nets, n, e, slots;
    int mx_n, mx_e;  // the largest net's nodes and parent edges
};

// Detour DAGs built on the device (dagbuild.cu) for a list of routing nets,
// placed in node, edge and point pools.  DAGs that outgrow a thread's work
// area are built again with larger slices; DAGs that find a pool full are
// built again after the pools have grown (keeping what they hold).
struct DeviceDags {
    DevBuf<int> work, sizes, list;
    DevBuf<long long> node_at, edge_at, point_at;
    DevBuf<unsigned long long> used;
    DevBuf<int> nodes, par_num, child_num, depth, par, child_idx, points;
    double per_node = 64, per_edge = 80, per_point = 48;  // entries per DAG of the last build
    std::vector<int> hs;    // [k][kDagSizeFields] after build()
    std::vector<int> tier;  // work-area size class each DAG fits
    // a.ids, a.n_list and the tree, congestion and grid fields set; the rest
    // is filled in here
    // order_key (optional, per DAG): the first class builds its DAGs in
    // descending key order
    void build(DagBuildArgs a, cudaStream_t s, const std::vector<int> *order_key = nullptr);
    int sz(int k, int f) const { return hs[(size_t)k * kDagSizeFields + f]; }
};

// Device arrays of one routing grid (build_cuda_database, database_cuda.hpp:2096-2362).
struct GridOwner {
    GridDev g;
    DevBuf<float> cap, demand, vcost;
    DevBuf<double> presum;
    DevBuf<int> pre, stamp, xlen, ylen, err;
    DevBuf<double> short_cost, score;
    DevBuf<uint8_t> dirty_cost, dirty_commit;
    DevBuf<unsigned long long> stats;
    std::vector<int> layer_first;
    // L, X, Y, DIR, edge lengths, unit costs, short costs [L], capacity [l][x][y] in reference layout
    void create(int L, int X, int Y, int DIR, const int *xlen, const int *ylen, double unit_wire, double unit_via,
                const double *short_cost, const float *cap_ref, cudaStream_t s);
    void reset_demand(cudaStream_t s);  // zero demand/pre/stamp/stats, mark all tracks dirty
    void mark_all_dirty(cudaStream_t s);
    int check_error(cudaStream_t s);    // device error word -> status (and clears it)
};

struct RouterStats {
    double wall = 0, p1_ms = 0, rrr_ms = 0, dag_host_ms = 0;
    int batches1 = 0, rerouted = 0;
    long long launches = 0;
    long long h2d_bytes = 0, d2h_bytes = 0;
    long long color_rounds = 0;
};

// Per-kernel-class device time, measured with CUDA events around each launch
// when profiling is on.
enum KernelClass {
    KC_COST = 0, KC_PATTERN, KC_WIRE_COMMIT, KC_VIA_COMMIT, KC_DAG, KC_COLOR, KC_RIPUP, KC_GRAPH1, KC_COMMIT_REFRESH, KC_N
};
struct KernelTimer {
    bool on = false;
    cudaStream_t s = nullptr;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[KC_N];
    double ms[KC_N] = {0};
    long long launches[KC_N] = {0};
    void begin(int k);
    void end(int k);
    void collect();  // after a stream synchronisation
    void reset();
};

// Conflict shapes of a set of nets for the batch colouring, in shape order.
struct ShapeSet {
    std::vector<int> pt_off{0}, pts, pt_net, h_off{0}, hseg, v_off{0}, vseg;
};
struct ShapeDev {
    DevBuf<int> pt_off, pts, pt_net, h_off, hseg, v_off, vseg, claim_off, claim;
    DevBuf<int> pt_n, claim_n;  // distinct points / claims per shape (shapes built on the device)
    int npts = 0, nshapes = 0, sparsity = 0;
    int64_t bytes = 0;  // host-to-device bytes of the last upload
    void upload(const ShapeSet &s, int X, int Y, int sparsity, cudaStream_t st, int threads = 0);
};

struct SeedModel;

// result of a run kept aside while another run is made (seeded against plain)
struct RouteBackup {
    DevBuf<int> routes;
    DevBuf<float> demand;
    std::vector<int64_t> route_off;
    std::vector<int> route_cap;
    int64_t route_end = 0;
    RouterStats st;
    std::vector<double> kt_ms;
    double score[3] = {0, 0, 0};
    unsigned long long cost_cells = 0, commit_cells = 0, commit_refresh_cells = 0;
    double color_bytes = 0;
};

struct Router {
    int rrr_iters = 1, threads = 0, mode = -1, verbose = 0, batched = 0;
    int split_commit = 0;  // 1: separate cost refresh, wire commit and via commit launches per phase-1 batch
    int host_dags = 0;     // 1: detour DAGs and batch arrays of the rip-up passes built on host threads
    Design d;
    NetSet ns;
    GridOwner go;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // batched form: the large and small size classes run beside the medium one
    // on these streams, forked from and joined back into `s`
    cudaStream_t s_cls[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    // the DAG gather of a pass's later batches runs on s_cls[1] beside the
    // first batch; batch 1 waits for ev_gjoin
    cudaEvent_t ev_gfork = nullptr, ev_gjoin = nullptr;
    bool gather_pending = false;
    RouterStats st;
    KernelTimer kt;
    int global_stamp = 0;
    int mode_eff = 0;

    // ---- inputs resident in HBM after open(): trees and conflict shapes in net-id order
    std::vector<int> tree_off;                                    // DFS preorder (Lshape_route.hpp:191-208)
    std::vector<int, NoInitAlloc<int>> tree_nodes, tree_par;
    std::vector<int64_t> scratch_off;                  // per net: DP scratch offset, -1 = on chip
    std::vector<int> order1;                           // phase-1 priority order (HPWL descending)
    int64_t scratch_nodes = 0;
    DevBuf<int> d_tree_off, d_tree_nodes, d_tree_par;
    DevBuf<int64_t> d_scratch_off;
    DevBuf<double> d_scratch;
    ShapeDev d_shapes1;
    // conflict shapes of a rip-up pass's nets: kept by the router, so that its
    // grow-only buffers serve every pass and run without new allocations
    ShapeDev d_shapes2;
    // ---- route records: phase-1 records at fixed offsets, reroutes appended per run
    std::vector<int64_t> route_off, route_off1;
    std::vector<int> route_cap, route_cap1;
    int64_t route_end1 = 0, route_end = 0;
    bool ran = false;
    DevBuf<int> routes;
    DevBuf<int64_t> d_route_off, d_old_off, d_slots;
    DevBuf<int> d_route_cap;
    // host copy of the live route records, packed on the device and made on
    // demand: page-locked ...
    PinnedBuf<int> h_routes;
    std::vector<int> h_routes_pageable;  // ... or, for a large first copy, pageable
    const int *h_routes_ptr = nullptr;
    std::vector<int64_t> h_route_at;     // [R+1] record of each routing net in the host copy
    bool h_routes_valid = false;
    DevBuf<int64_t> d_dense_off;
    DevBuf<int> d_dense;
    // ---- per-run device buffers (grow-only)
    DevBuf<int4> d_hdr;
    DevBuf<int> d_vcnt;  // via crossings per cell of the current phase-1 batch (fused commit)
    DevBuf<unsigned long long> d_cops;  // colouring operation counts of the current run
    double color_bytes = 0;             // algorithmic bytes of the colouring kernels of the last run
    double dp_bytes = 0;                // algorithmic bytes of one phase-1 tree DP pass
    int64_t setup_h2d = 0;              // host-to-device bytes of the device setup
    DevBuf<int> d_ids, d_all_ids, of_sum, d_perm, d_map, d_bat, d_act, d_flags, d_queue;
    DevBuf<int> d_rev_off, d_rev_cnt, d_rev, d_snap, d_dirty, d_part;  // colouring: claimers per cell, round-0 map
    // launch shape of the tree DP per size class (large, medium, small) and the
    // node count that separates small from medium nets (autotuned, see tune.cpp)
    struct Tune {
        int classes = 1;  // 1: one DP launch per batch (largest nets first); 3: large/medium/small launches
        int split = 6;
        int lanes[3] = {32, 32, 16};
    } tune;
    bool tuned = false;
    DevBuf<int64_t> d_route_off1;
    DevBuf<int> d_route_cap1;
    // phase-1 loop captured as a CUDA graph (batched form) and the plan it was captured for
    cudaGraphExec_t graph1_exec = nullptr;
    std::vector<int> graph1_batch_off, graph1_class_off;
    int *graph1_routes = nullptr;
    int graph1_seed = 0;  // seeding of the captured loop (0 none, 1 + decay levels)
    long long graph1_launches = 0;
    // device plan of phase 1 from the colouring in d_bat (ranks of d_perm1):
    // d_ids, and the batch and class offsets on the host
    void plan_phase1(int nb, std::vector<int> &batch_off, std::vector<int> &class_off);
    void emit_phase1(const std::vector<int> &batch_off, const std::vector<int> &class_off, bool timed);
    void autotune(int nb);
    DevBuf<int> d_perm1, d_plan_hist, d_plan_offs;  // phase-1 colouring ranks, plan scratch
    DevBuf<uint8_t> d_is_of;
    DevBuf<float> d_xsum, d_ysum;
    DevBuf<int> dg_nodes, dg_paroff, dg_par, dg_cslot, dg_echild, dg_childoff, dg_leveloff, dg_levelnodes, dg_nno,
        dg_netlvl, dg_ids, dg_bchange, dg_lout, dg_stage, dg_scnt;
    DevBuf<double> dg_costs, dg_cedges, dg_offers;
    DevBuf<unsigned long long> dg_best, dg_packed;
    // arenas of the DAG arrays (declared before the DAGs: freed after them)
    std::vector<std::unique_ptr<std::pmr::monotonic_buffer_resource>> dag_arenas;
    std::vector<DagNet> dag;     // detour DAGs of the nets rerouted in the current pass
    std::vector<int> dag_slot;   // routing net -> its DAG in `dag`, -1 when not rerouted
    unsigned long long cost_cells = 0, commit_cells = 0, commit_refresh_cells = 0;
    // phase-1 plan of the last run (routing order, batches, trees, route capacity in order)
    std::vector<int> plan_ids, plan_batch_off, plan_node_off, plan_nodes, plan_par, plan_cap;
    bool plan_built = false;
    void build_plan();
    // score of the last run: wirelength, vias, overflow (GPU estimate)
    double score_wl = 0, score_via = 0, score_of = 0;
    int64_t pin_vias = -1;  // selected pins on file layer 0 (one via each), counted once

    // learned congestion seed (not owned): 1 = seeded runs, 2 = seeded run
    // judged against a plain run (the better score is kept)
    SeedModel *seed = nullptr;
    double seed_alpha = 0.5;
    int seed_mode = 0;
    int seed_kind = 0;    // 0 predicted demand, 1 predicted overflow only
    bool seed_order = false;  // rip-up order by predicted overflow instead of HPWL
    int seed_levels = 0;  // 0 constant during phase 1, else shrinks in this many steps
    bool seed_ready = false, seed_active = false, seed_used = false, seed_score_due = false;
    double seed_ms = 0, seed_scores[2] = {0, 0};
    DevBuf<float> d_seed_dem;         // seed demand at full strength (unrounded), track layout
    DevBuf<float> d_seed_cur;         // seed demand currently added to the demand (half units)
    std::vector<double> seed_sat;     // summed-area table of the predicted overflow
    std::vector<int> hpwl_keys;       // HPWL of every routing net, contiguous (rip-up order keys)
    void prepare_seed();
    // the seed's input features ([X][Y][16] bf16) on the device from the
    // resident trees (seed_feat.cu); synchronous on `st`
    void device_seed_features(DevBuf<__nv_bfloat16> &feat, cudaStream_t st);
    void seed_begin();
    double seed_pressure(int net) const;
    void seed_stats(double out[4]);  // [0] seeded result kept, [1] seeded score, [2] plain score, [3] prediction ms
    void run_once(bool seeded);
    void save_result(RouteBackup &b);
    void restore_result(RouteBackup &b);

    ~Router();
    void open(const char *cap, const char *net);
    void run();
    void write(const char *out);
    // Scores the last run with the ISPD2024 evaluator's rules on the device
    // (run/evaluator.cpp:462-633): out = {wirelength cost, via cost, overflow
    // cost, total}; layer_loss (optional, L entries) = overflow loss per routing layer.
    void evaluate(double *out, double *layer_loss);
    DevBuf<int64_t> ev_sel_off, ev_extra_off, ev_route_off;
    DevBuf<int> ev_sel, ev_extra, ev_sub_off, ev_wire, ev_stacked;
    DevBuf<long long> ev_vcnt, ev_ccnt, ev_voff;
    DevBuf<unsigned long long> ev_cnt, ev_wkeys, ev_vkeys, ev_vloc;
    DevBuf<unsigned> ev_vfirst, ev_vord;
    DevBuf<double> ev_part, ev_capd, ev_capd_ref;
    void fetch_routes();
    const int *route_of(int net) const { return h_routes_ptr + h_route_at[net]; }
    void ensure_device();
    void device_shapes(const ShapeArgs &a, ShapeDev &sd);
    DevBuf<long long> d_shape_tot;
    DevBuf<int> d2_ptoff, d2_pts, d2_ids;  // DAG points and net ids of the rerouted nets
    // device DAG construction: trees in adjacency order (positions, neighbour
    // lists), the builder, kept nets and the batch layout of the gather
    DevBuf<int> d_dt_off, d_dt_pos, d_dt_aoff, d_dt_adj, d_kept, d_kept_dag, d_gdesc, d_gbatch;
    DevBuf<int> d_of_list, d_of_blocks;  // nets flagged for rip-up (id order), list scratch and count
    DevBuf<long long> d2_extat;
    bool dt_ready = false;
    DeviceDags ddag;
    // stream, events and the routing grid on the device; started on a thread of
    // its own by open() as soon as the capacities are read
    void create_grid();
    void join_grid();
    std::thread grid_thread;
    std::exception_ptr grid_err;
    bool grid_ready = false, device_ready = false;
    double ctx_seconds = 0;  // context creation on the side thread (verbose report)
    void color_nets(const std::vector<int> &order, const ShapeDev &shapes, int sparsity,
                    std::vector<std::vector<int>> &batches);
    // colours n ranks (d_perm_ranks[k] = shape of rank k) into d_bat; returns the batch count
    int run_color(int n, const int *d_perm_ranks, const ShapeDev &shapes, int sparsity);
    void compute_score();
    // detour DAGs of the rerouted nets built, coloured and laid out per batch
    // on the device; false when no net is left to reroute.  tm: times at which
    // the DAGs, conflict shapes, colouring and batch arrays were done
    std::vector<int> pass_order(const std::vector<int> &of_ids) const;
    bool dags_on_device(std::vector<int> &of_nets, std::future<std::vector<int>> &order,
                        std::vector<std::vector<int>> &batches,
                        std::vector<DagBatchInfo> &bi, const std::vector<int64_t> &old_off, double *tm);
    void upload_dag_trees();  // trees in adjacency order, once per router (enqueued, no sync)
    // the trees in adjacency order packed into page-locked buffers; the first
    // run packs them on a side thread while phase 1 runs on the device
    struct PackedTrees {
        int *off = nullptr, *pos = nullptr, *aoff = nullptr, *adj = nullptr;
        size_t n_off = 0, n_pos = 0, n_aoff = 0, n_adj = 0;
        PackedTrees() = default;
        PackedTrees(const PackedTrees &) = delete;
        PackedTrees &operator=(const PackedTrees &) = delete;
        ~PackedTrees() { release(); }
        void release();  // back to the page-locked block cache
    };
    PackedTrees dt_pack;
    std::future<void> dt_packing;  // declared after the trees it reads: joined first on destruction
    // the phase-1 priority order, sorted on a host thread from open() on (it
    // reads hpwl_keys); taken into order1 where the device setup needs it
    std::future<std::vector<int>> order1_pending;
    void pack_dag_trees();

   private:
    void phase1();
    bool rrr_pass(int iter);
    void grow_routes(int64_t need);
};

}  // namespace igr
