// Device state of the router and the launchers of its sm_100a kernels.
//
// Grid arrays are per routing layer and track-contiguous: on a vertical layer
// (tracks run along y) cell (l, x, y) lives at l*X*Y + x*Y + y, on a
// horizontal layer (tracks run along x) at l*X*Y + y*X + x.  Every track is
// therefore one contiguous run, so the per-track passes (cost refresh with its
// prefix sums, difference-array commit, overflow scans) stream it with
// coalesced loads.  Route records keep InstantGR's position encoding
// l*X*Y + x*Y + y so that they can be exchanged with it unchanged.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "status.hpp"

namespace igr {

// longest track: the reference's compute_presum holds a track in at most
// 120 KB of shared memory, 15,360 doubles (src/main.cpp:28)
constexpr int kMaxTrackCells = 15360;
// longest track of the fused batch commit (commit_refresh); grids with longer
// tracks commit with the separate wire and via launches
constexpr int kMaxFusedTrackCells = 4096;

constexpr int kStatSlots = 5;  // entries of GridDev::stats

struct GridDev {
    int L = 0, X = 0, Y = 0, DIR = 0;  // routing layers, grid, direction of routing layer 0
    int64_t N = 0;                      // L*X*Y cells
    int ntracks = 0;                    // sum over layers of (X or Y)
    double unit_wire = 0, unit_via = 0;
    // device arrays
    float *cap = nullptr, *demand = nullptr, *vcost = nullptr;
    double *presum = nullptr;
    int *pre = nullptr;        // wire difference array (zero between batches)
    int *stamp = nullptr;      // timestamp per cell
    int *xlen = nullptr, *ylen = nullptr;
    double *short_cost = nullptr;  // [L]
    uint8_t *dirty_cost = nullptr;    // [ntracks] demand changed since the last cost refresh
    uint8_t *dirty_commit = nullptr;  // [ntracks] difference array holds entries
    unsigned long long *stats = nullptr;  // [0] wirelength, [1] via count (signed, two's complement),
                                          // [2] cells refreshed by cost_refresh, [3] cells committed and
                                          // [4] cells refreshed by commit_refresh
    int *err = nullptr;                   // device error word
};

// track id of layer l, track index t (y for horizontal layers, x for vertical)
struct TrackMap {
    std::vector<int> first;  // [L+1] first track id of each layer
};

// Launch set-up of one kernel that is a per-device setting: the dynamic
// shared-memory limit (raised to the largest `smem` asked for so far), the SM
// count and the resident blocks per SM for `threads` threads and `smem` bytes.
// Done once per (kernel, device, smem) under a lock, so that contexts on
// several devices and host threads each get their own; a failing CUDA call
// throws igr::Error (ERR_CUDA).
struct KernelShape {
    int sms = 0;
    int blocks_per_sm = 0;
};
KernelShape kernel_setup(const void *kernel, int threads, size_t smem);

// ---- launchers (stream-ordered; errors are reported through cudaGetLastError)
void launch_cost_refresh(const GridDev &g, bool only_dirty, cudaStream_t s);
void launch_wire_commit(const GridDev &g, int stamp, bool only_dirty, cudaStream_t s);
// Commit of a tree-DP batch (wires from the difference array, vias from the
// per-cell crossing counts `vcnt`, which it clears) and cost refresh, fused per
// track; refresh = false only commits and marks the costs dirty.
void launch_commit_refresh(const GridDev &g, int *vcnt, int stamp, bool refresh, cudaStream_t s);

struct TreeBatchDev {
    const int *net_ids;      // [n] routing-net id of each net of the batch
    const int *node_off;     // [routing nets+1] node offset of each net id (into nodes/par)
    const int *nodes;        // tree nodes, preorder, reference encoding (Steiner layer = L)
    const int *par;          // parent (local index) per node, -1 at the root
    const int64_t *route_off;  // [routing nets] route record offset (ints)
    const int *route_cap;    // [routing nets] route record capacity (ints)
    int *routes;             // route records
    double *scratch;         // per-node DP tables of nets larger than the shared-memory tile
    const int64_t *scratch_off;  // [routing nets] offset (in nodes) into scratch, -1 for nets that fit on chip
    int64_t scratch_nodes;   // nodes covered by scratch: kPatternScratchD doubles each, then kPatternScratchI ints each
    int n;
    const int *order = nullptr;  // [n] positions into net_ids in processing order (null: 0..n-1)
    int *queue = nullptr;        // work counter of this launch (zero before the launch)
    int lanes_per_net = 32;      // 16 or 32
    int tile = 16;               // nodes kept on chip: 6, 16, 32, or 1 (all in scratch)
    int *vcnt = nullptr;         // non-null: count via crossings per cell here (and the via
                                 // count in stats[1]) for launch_commit_refresh
};
// scratch per node of a net kept in global memory: 45 range costs (doubles),
// then 8 via-column costs (floats), 45 backtrace codes (shorts, padded to 23
// ints), the chosen range and 4 decoded position/parent ints
constexpr int kPatternScratchD = 45, kPatternScratchI = 8 + 23 + 1 + 4;
// doubles of scratch needed for `nodes` nodes of nets kept in global memory
inline int64_t pattern_scratch_doubles(int64_t nodes) {
    return nodes * kPatternScratchD + (nodes * kPatternScratchI + 1) / 2;
}
constexpr int kPatternNodeTile = 16;  // nets with more nodes use global scratch
void launch_pattern_route(const GridDev &g, const TreeBatchDev &b, int stamp, cudaStream_t s);

// Tree DP over caller-owned device arrays with its scratch in a fixed array of
// the library's device image (pattern_static.cu); synchronous on `s`.
constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kStaticMaxNets = 1 << 20;
constexpr int kStaticMaxDevices = 64;
void pattern_route_static(const GridDev &g, int n, const int *node_off, int64_t total_nodes, const int *nodes,
                          const int *par, const int64_t *route_off, const int *route_cap, int *routes,
                          int64_t routes_len, int stamp, cudaStream_t s);

struct ViaBatchDev {
    const int *net_ids;  // [n]
    const int64_t *route_off;
    const int *routes;
    int n;
};
void launch_via_commit(const GridDev &g, const ViaBatchDev &b, int stamp, int K, cudaStream_t s);
void launch_wire_ripup(const GridDev &g, const ViaBatchDev &b, int stamp, int K, cudaStream_t s);

// Batch of detour DAGs (phase 2).  Node indices are batch-global; the parent
// slots of node v are par_off[v]..par_off[v+1] (edge e: parent par[e], child
// slot child_slot[e] of the parent, child node edge_child[e]); the child slots
// of v are child_off[v]..child_off[v+1].
struct DagBatchDev {
    int n_nodes = 0, n_edges = 0, n_nets = 0;
    const int *nodes = nullptr, *par_off = nullptr, *par = nullptr, *child_slot = nullptr, *edge_child = nullptr;
    const int *child_off = nullptr;
    // levels of each net (dag_levels): net k's levels are level_off[net_level_off[k] + d],
    // d = 0..depth_k, positions into level_nodes
    const int *level_off = nullptr, *level_nodes = nullptr, *net_level_off = nullptr;
    const int *net_node_off = nullptr, *net_ids = nullptr;
    double *costs = nullptr;
    unsigned long long *best_path = nullptr, *packed = nullptr;
    double *cost_edges = nullptr;
    int *best_change = nullptr, *layer_out = nullptr, *stage = nullptr, *stage_cnt = nullptr;
    const int64_t *route_off = nullptr;
    const int *route_cap = nullptr;
    int *routes = nullptr;
    // the batch's largest net in nodes and in parent edges (0: not known);
    // they size the shared memory that stages a net's DAG
    int max_net_nodes = 0, max_net_edges = 0;
    // 54 doubles per parent edge: the offer records of staged nets (null: no
    // net is staged)
    double *offers = nullptr;
};
// per-net level lists of n nets whose nodes are node_off[k]..node_off[k+1]:
// level_nodes holds each net's nodes by depth (stable), level_off the depth_k + 1
// level boundaries of each net, net_level_off[k] where net k's boundaries start
void dag_levels(int n, const int *node_off, const int *depth, std::vector<int> &level_nodes,
                std::vector<int> &level_off, std::vector<int> &net_level_off);
// edge costs, then one CTA per net; returns the number of kernel launches
// aux, fork, join (optional): in batches of 4096 nets or more, the DAGs of
// more than 64 nodes run on `aux` beside the smaller ones
// Batches of `split_nets` nets or more (4096 by default) run the DAGs of at
// most 64 nodes in 2-warp CTAs on `s` beside the larger ones on `aux`
// (forked and joined through the two events); smaller batches, or no `aux`,
// run one launch, or (with `aux`, when the batch holds DAGs of more than 96
// nodes) the DAGs of at most 96 nodes on `s` beside the larger ones on `aux`.
// Nets of at most `stage_nodes` nodes (0: none) whose DAG fits a CTA's shared
// memory keep it there while they are routed.
int launch_dag_route(const GridDev &g, const DagBatchDev &b, int stamp, cudaStream_t s, cudaStream_t aux = nullptr,
                     cudaEvent_t fork = nullptr, cudaEvent_t join = nullptr, int split_nets = 4096,
                     int stage_nodes = 1024);

constexpr int kRouteLayers = 9;

// rip-up marking (graph.hpp:432-466): flags nets whose routes cross more than
// `min_edges` edges with cap + threshold <= demand
void launch_mark_overflow(const GridDev &g, int threshold, int *of_sum, const ViaBatchDev &nets,
                          int min_edges, uint8_t *is_of, cudaStream_t s);
// indices i < n with flags[i] set, increasing, into list[0..*count); block_cnt
// holds flag_list_blocks(n) ints of scratch
int flag_list_blocks(int n);
void launch_flag_list(const uint8_t *flags, int n, int *list, int *count, int *block_cnt, cudaStream_t s);
// 2-D congestion view (graph.hpp:545-584): max over layers of (demand - cap)^+, then
// exclusive prefix sums along x (xsum) and along y (ysum); layout [x][y]
void launch_congestion_view(const GridDev &g, float *xsum, float *ysum, cudaStream_t s);
// overflow cost of the current demand (graph.hpp:148-157), summed in fixed order
void launch_overflow_cost(const GridDev &g, double *out, cudaStream_t s);

// layout conversions between the reference layout [l][x][y] and the track layout
void launch_to_track_layout(const GridDev &g, const float *ref, float *trk, cudaStream_t s);
void launch_from_track_layout_f(const GridDev &g, const float *trk, float *ref, cudaStream_t s);
void launch_from_track_layout_d(const GridDev &g, const double *trk, double *ref, cudaStream_t s);
void launch_to_track_layout_d(const GridDev &g, const double *ref, double *trk, cudaStream_t s);
void launch_from_track_layout_i(const GridDev &g, const int *trk, int *ref, cudaStream_t s);
void launch_to_track_layout_i(const GridDev &g, const int *ref, int *trk, cudaStream_t s);

// ---- conflict shapes and claim lists from the flattened trees (shapes.cu).
// Shape k is routing net ids[k] (k when ids is null); its points are its tree's
// nodes and edge points, or ext_pts[ext_off[k] .. ext_off[k+1]) when ext_off is
// given; its segments are its tree's.  Counts and offsets first (pt_off,
// claim_off: [n+1]; totals: points, claims), then the fill.
struct ShapeArgs {
    const int *tree_off = nullptr, *tree_nodes = nullptr, *tree_par = nullptr;
    const int *ids = nullptr, *ext_off = nullptr, *ext_pts = nullptr;
    // instead of ext_off: shape k's points start at ext_at[k], ext_cnt[k * ext_stride] of them
    const long long *ext_at = nullptr;
    const int *ext_cnt = nullptr;
    int ext_stride = 1;
    int n = 0, X = 0, Y = 0, sparsity = 15;
};
void launch_shape_count(const ShapeArgs &a, int *pt_off, int *claim_off, long long *totals, cudaStream_t s);
// pt_n / claim_n (optional, [n]): per shape the number of distinct points and
// claimed cells, which the fill sorts and moves to the front of each range
void launch_shape_fill(const ShapeArgs &a, const int *pt_off, const int *claim_off, int *pts, int *claim,
                       int *pt_n, int *claim_n, cudaStream_t s);

// ---- detour DAGs on the device (dagbuild.cu)
// slice sizes of one builder thread's work area: tree nodes, stem entries,
// mirror entries, DAG nodes, links, conflict points (before deduplication)
struct DagCaps {
    int tc = 32, sc = 512, mc = 512, nc = 512, ec = 1024, pc = 2048;
};
constexpr int kDagSizeFields = 7;  // per DAG: nodes, links, points, depth levels, child slots, widest slot, status
struct DagBuildArgs {
    int n_list = 0;
    const int *list = nullptr;      // DAGs to build (positions k); null: 0..n_list-1
    const int *ids = nullptr;       // [k] routing net of DAG k
    const int *tree_off = nullptr;  // [R+1] tree nodes of each routing net, in adjacency order
    const int *pos = nullptr;       // tree node positions (3-D; Steiner nodes on layer 9)
    const int *adj_off = nullptr;   // [tree nodes + 1] neighbour list of each tree node
    const int *adj = nullptr;       // neighbours (net-local indices)
    const float *xsum = nullptr, *ysum = nullptr;  // congestion view [X][Y]
    int X = 0, Y = 0, mode = 2;
    DagCaps caps;
    int *work = nullptr;            // threads x dag_work_ints(caps)
    int *sizes = nullptr;           // [k][kDagSizeFields]; status 1: work area too small, 2: malformed, 3: pool full
    long long *node_at = nullptr, *edge_at = nullptr, *point_at = nullptr;  // [k] where DAG k was placed
    // pools: entries used so far (nodes, edges, points) and their capacities
    unsigned long long *used = nullptr;
    long long cap_nodes = 0, cap_edges = 0, cap_points = 0;
    int *out_nodes = nullptr, *out_par_num = nullptr, *out_child_num = nullptr, *out_depth = nullptr;
    int *out_par = nullptr, *out_child_idx = nullptr, *out_points = nullptr;
};
long long dag_work_ints(const DagCaps &c);
void launch_dag_build(const DagBuildArgs &a, int threads, cudaStream_t s);
// one builder per block: work area in shared memory (a.work null, at most
// dag_solo_smem_limit() bytes) or in global memory (builders x slices)
void launch_dag_build_solo(const DagBuildArgs &a, int builders, cudaStream_t s);
int dag_solo_smem_limit();
// batch layout: per net (in batch order) its DAG k, batch-local node base,
// edge base, slot base, level base, position in the batch and batch; per
// batch its first node, edge, node+1, level and net entries and first net
constexpr int kDagDescFields = 7;
constexpr int kDagBatchFields = 6;
struct DagGatherArgs {
    int n = 0;
    const int *desc = nullptr, *batch = nullptr, *ids = nullptr, *sizes = nullptr;
    const long long *node_at = nullptr, *edge_at = nullptr;
    const int *src_nodes = nullptr, *src_par_num = nullptr, *src_child_num = nullptr, *src_depth = nullptr;
    const int *src_par = nullptr, *src_child_idx = nullptr;
    int *nodes = nullptr, *par_off = nullptr, *par = nullptr, *child_slot = nullptr, *edge_child = nullptr,
        *child_off = nullptr, *level_off = nullptr, *level_nodes = nullptr, *net_node_off = nullptr,
        *net_ids = nullptr, *net_level_off = nullptr;
};
void launch_dag_gather(const DagGatherArgs &a, cudaStream_t s);

// ---- dense copy of the live route records (records.cu): record lengths and
// their exclusive scan into off[0..n] (off: [n+1]), then the copy into dense
void launch_record_offsets(const int *routes, const int64_t *route_off, int n, int64_t end, int64_t *off,
                           cudaStream_t s);
void launch_record_copy(const int *routes, const int64_t *route_off, int n, const int64_t *off, int *dense,
                        cudaStream_t s);
// record slots of n nets: route_off[id] = offset and route_cap[id] = capacity
// for slot[3k .. 3k+2] = {id, offset, capacity}
void launch_record_slots(int n, const int64_t *slot, int64_t *route_off, int *route_cap, cudaStream_t s);
// dst[k] = src[idx[k]], k < n
void launch_take_i64(int n, const int *idx, const long long *src, long long *dst, cudaStream_t s);

// ---- evaluation of a routing result with the ISPD2024 evaluator's rules (eval.cu)
constexpr int kEvalLayers = 10;  // file layers: 0 (pins) and the 9 routing layers
struct EvalDev {
    int n = 0, L = 0, X = 0, Y = 0, DIR = 0;      // design nets, routing layers, grid
    const int64_t *sel_off = nullptr, *extra_off = nullptr;  // pins and stacked-pin pairs per design net
    const int *sel = nullptr, *extra = nullptr;   // file-layer 3-D positions
    const int *sub_off = nullptr;                 // [n+1] routing nets of each design net
    const int64_t *route_off = nullptr;           // route record of each routing net
    const int *routes = nullptr;
    const float *cap = nullptr;                   // routing-layer capacity (track layout)
    const double *cap_d = nullptr;                // the same in double where a value is not a float
    const int *xlen = nullptr, *ylen = nullptr;   // GCell widths along x and y
    int *wire = nullptr, *stacked = nullptr;      // per routing cell (track layout)
    unsigned long long *total_vias = nullptr;     // [kEvalLayers]
    unsigned long long *wl = nullptr;             // [L] wire length per routing layer
    unsigned long long *wkeys = nullptr, *vkeys = nullptr;  // hash sets of wire cells and via locations
    unsigned long long wmask = 0, vmask = 0;      // table sizes - 1 (powers of two)
    unsigned *vfirst = nullptr;                   // first position of each via location (by slot)
    unsigned long long *vloc = nullptr;           // via locations in order
    unsigned *vord = nullptr;                     // their line positions
    int *err = nullptr;
};
void launch_eval_count(const EvalDev &e, long long *via_cnt, long long *cell_cnt, cudaStream_t s);
void launch_eval_marks(const EvalDev &e, const long long *via_off, long long nloc, cudaStream_t s);
int eval_blocks_per_layer(int64_t XY);
// per (routing layer, block) overflow-loss partial sums into part[L * blocks]
void launch_eval_cells(const EvalDev &e, int blocks_per_layer, double *part, cudaStream_t s);

// ---- phase-1 plan from the colouring (plan.cu): routing-net ids batch by
// batch in routing order (batches reversed), each batch split into the size
// classes of the tree DP, nets of a class by node count (largest first)
struct PlanArgs {
    int n = 0, nb = 0;                // ranks, batches
    const int *bat = nullptr;         // [n] batch of each rank
    const int *perm = nullptr;        // [n] routing-net id of each rank (null: identity)
    const int *node_off = nullptr;    // [routing nets+1] tree node offsets
    int classes = 1, split = 6, big = 16;  // 1 class (all medium), or large (> big) / medium (> split) / small
};
// histogram entries launch_plan needs for nb batches
int64_t plan_hist_size(int nb);
// ids[n]; offs[3 * rb + c] = first position of class c of routed batch rb, offs[3 * nb] = n
void launch_plan(const PlanArgs &a, int *hist, int *ids, int *offs, int *err, cudaStream_t s);

// ---- batch colouring (database_cuda.hpp:288-434, made deterministic)
struct ColorDev {
    int n = 0, X = 0, Y = 0, sparsity = 15;
    // shapes are indexed by shape id s; the colouring ranks k = 0..n-1 (higher
    // k wins a cell) with perm[k] = shape of rank k (null: identity)
    const int *perm = nullptr;
    const int *pt_off = nullptr, *pts = nullptr;   // [shapes+1], 2-D cells
    const int *pt_net = nullptr;                   // [points] owner shape
    const int *h_off = nullptr, *hseg = nullptr;   // [shapes+1], pairs
    const int *v_off = nullptr, *vseg = nullptr;
    // cells claimed by each shape: 4-neighbourhood of its points, every
    // `sparsity`-th cell of its segments (CSR over shapes)
    const int *claim_off = nullptr, *claim = nullptr;
    // optional [shapes]: the shape's distinct claims / points are the first
    // claim_n[s] / pt_n[s] entries of its range (else the whole range)
    const int *claim_n = nullptr, *pt_n = nullptr;
    int npts = 0;
    int *map = nullptr;       // [X*Y]
    int *batch = nullptr;     // [n]
    // net lists, [n] each: nets without a batch (two buffers), candidates of a
    // round, nets that lost a point in a round
    int *active = nullptr, *active2 = nullptr, *cand = nullptr, *lost = nullptr;
    int4 *hdr = nullptr;      // [n] per rank: claim begin/end, point begin/end
    // optional [5] operation counts, accumulated: claimed cells, commit point
    // checks, blocking point checks, release checks, list entries scanned
    unsigned long long *ops = nullptr;
    int *flags = nullptr;     // [16] device flags
    int rounds = 0;           // out: colouring rounds run
    // optional (all or none): the round-0 map of every batch kept up to date
    // instead of re-claimed.  rev_off/rev_cnt [X*Y]: claimers of each cell in
    // rev[] (ranks; [total claims]); snap/dirty [X*Y]; part [1024]
    int *rev_off = nullptr, *rev_cnt = nullptr, *rev = nullptr, *snap = nullptr, *dirty = nullptr, *part = nullptr;
    // bound of every grid-barrier wait, and arrivals it waits for that never
    // come (test hook; run_coloring takes both from the process's test hooks)
    unsigned long long wait_ns = 2000000000ull;
    unsigned phantom = 0;
};
// Claim lists of shapes (pt_off/pts/h_off/hseg/v_off/vseg as in ColorDev).
void build_claims(int nshapes, const int *pt_off, const int *pts, const int *h_off, const int *hseg,
                  const int *v_off, const int *vseg, int X, int Y, int sparsity, std::vector<int> &off,
                  std::vector<int> &cells, int threads);
int run_coloring(ColorDev &c, int max_batch, cudaStream_t s);  // returns #batches (host loop)

std::string cuda_error_string(cudaError_t e);

}  // namespace igr
