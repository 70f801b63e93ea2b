/*
 * instantgr_b200 — C ABI of a B200-native (sm_100a) GPU global router that is
 * a drop-in for InstantGR's routing hot path.
 *
 * Two levels:
 *   1. The router: the whole `-cap <f> -net <f> -out <f>` flow of InstantGR
 *      (src/main.cpp:91-102, route() at :22-73) behind igr_route_files and
 *      the igr_router_* calls, which a host program can drive stage by stage.
 *   2. The device operators of the hot path, one per kernel group of
 *      InstantGR, on an igr_ctx that owns all device state of one routing grid.
 *
 * Conventions
 *   - Every call returns 0 on success or a negative IGR_ERR_* code; the
 *     message of the last failure is returned by igr_last_error().  No call
 *     exits the process (InstantGR calls exit() on CUDA errors,
 *     src/Lshape_route_detour.hpp:1088-1091).
 *   - Positions use InstantGR's encoding pos = l*X*Y + x*Y + y, with l the
 *     routing layer (file layer - 1, src/database_cuda.hpp:2106).  Grid arrays
 *     passed in or out are in InstantGR's layout [l][x][y] (y fastest).
 *   - Calls on one context are ordered on its CUDA stream and must come from
 *     one host thread at a time.  Host buffers belong to the caller.
 *   - Route records are InstantGR's: int count c at [0] (the next free
 *     slot, so c = 1 + 2 * pairs), then c-1 ints of position pairs.
 */
#ifndef INSTANTGR_B200_H
#define INSTANTGR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IGR_OK 0
#define IGR_ERR_INVALID (-1)  /* bad argument */
#define IGR_ERR_IO (-2)       /* file could not be read or written */
#define IGR_ERR_FORMAT (-3)   /* malformed .cap/.net */
#define IGR_ERR_CUDA (-4)     /* CUDA runtime error (no device, launch failure, ...) */
#define IGR_ERR_CAPACITY (-5) /* a fixed-size buffer or limit was exceeded */
#define IGR_ERR_TIMEOUT (-6)  /* a bounded device wait gave up */
#define IGR_ERR_STATE (-7)    /* inconsistent input (e.g. a tree that is not in preorder) */

typedef struct igr_ctx igr_ctx;
typedef struct igr_router igr_router;

/* ------------------------------------------------------------------ router */

typedef struct igr_options {
    int rrr_iters;     /* rip-up-and-reroute iterations after phase 1 (InstantGR: 1) */
    int threads;       /* host threads, 0 = all cores */
    int mode;          /* DAG size mode of InstantGR (0..2); -1 = choose by net count as main.cpp:39-40 */
    int verbose;       /* print stage times to stderr */
    int batched;       /* 1 = size-class persistent kernels + CUDA graphs (same results as 0) */
    int profile;       /* 1 = time every kernel launch with CUDA events (igr_router_kstats) */
    int split_commit;  /* 1 = phase-1 batches commit wires and vias and refresh costs in three
                          launches instead of one fused per-track pass (same results) */
    int host_dags;     /* 1 = detour DAGs and the per-batch DAG arrays of the rip-up passes are
                          built on the host threads instead of the device (same results) */
    int reserved[5];
} igr_options;

/* Fills `o` with the defaults that reproduce InstantGR (1 RRR pass). */
void igr_default_options(igr_options *o);

/* Whole flow: read .cap/.net, route, write route guides.
 * Replaces `InstantGR -cap <cap> -net <net> -out <out>` (src/main.cpp:91-102). */
int igr_route_files(const char *cap_path, const char *net_path, const char *out_path, const igr_options *opt);

/* Stage-by-stage control of the same flow. */
int igr_router_open(const char *cap_path, const char *net_path, const igr_options *opt, igr_router **out);
/* Routes (or re-routes from empty demand): phase 1, then opt->rrr_iters
 * rip-up-and-reroute passes (src/main.cpp:22-73). */
int igr_router_run(igr_router *r);
/* Writes the route guides (src/graph.hpp:179-235). */
int igr_router_write(igr_router *r, const char *out_path);
/* Scores the last run on the device with the rules of the ISPD2024 evaluator
 * (run/evaluator.cpp:462-633, read_gr_solution), on the guides that
 * igr_router_write would write, without writing them: out[0] wirelength cost,
 * out[1] via cost, out[2] overflow cost, out[3] total (the evaluator's FOR_STAT
 * values before rounding); layer_loss[0..8] (may be null) the overflow loss of
 * each routing layer before its weight.  Connectivity is not checked (the
 * evaluator stops at the first open net instead of scoring).  No reference
 * counterpart in the router: it replaces running the evaluator on the file. */
int igr_router_evaluate(igr_router *r, double *out, double *layer_loss);
/* Statistics of the last run: [0] routing nets, [1] nets rerouted in the last
 * pass, [2] wirelength, [3] via count, [4] overflow cost (GPU estimate,
 * src/graph.hpp:148-169), [5] route wall seconds, [6] phase-1 batches,
 * [7] phase-1 device ms, [8] rip-up/reroute device ms, [9] host DAG ms,
 * [10] kernel launches, [11] design nets, [12] colouring rounds,
 * [13] host-to-device bytes, [14] device-to-host bytes (of the run and the
 * route download for writing), [15] host-to-device bytes of the one-time
 * device setup (grid, trees, conflict shapes). */
int igr_router_stats(igr_router *r, double *out, int n);
/* Per-kernel-class device time of the last run (needs opt->profile): for
 * class k in {cost refresh, tree DP, wire commit, via commit, DAG DP,
 * colouring, rip-up/marking, phase-1 graph, fused phase-1 commit and cost
 * refresh}, out[3k] = launches, out[3k+1] = milliseconds, out[3k+2] =
 * algorithmic DRAM bytes (cost refresh: 20 per refreshed cell; fused commit
 * and refresh: 20 per refreshed cell + 12 per committed cell;
 * colouring: 12 per claimed cell, 8 per commit point check, 12 per blocking
 * point check, 8 per release check, 8 per active-list entry scanned; tree
 * DP: 32 per node, 144 per straight and 360 per bent tree edge). */
int igr_router_kstats(igr_router *r, double *out, int n);
/* Phase-1 plan of the last run: routing order, batch offsets and trees.
 * sizes[0..2] receive the number of nets, batches and tree nodes; the arrays
 * (net_ids[n], batch_off[b+1], node_off[n+1], nodes[m], par[m], route_cap[n],
 * all in routing order) are filled when non-null. */
int igr_router_plan(igr_router *r, int64_t *sizes, int32_t *net_ids, int32_t *batch_off, int32_t *node_off,
                    int32_t *nodes, int32_t *par, int32_t *route_cap);
/* Grid of the design in the layout of igr_grid_desc: hdr = {L, X, Y, dir0},
 * costs = {unit_wire, unit_via, short_cost[L]}, edge lengths, capacity. */
int igr_router_grid(igr_router *r, int32_t *hdr, double *costs, int32_t *x_edge_len, int32_t *y_edge_len,
                    float *capacity);
/* Selects the CUDA device of the calling thread for subsequent calls. */
int igr_set_device(int device);
/* Number of design nets and routing nets. */
int igr_router_sizes(igr_router *r, int64_t *design_nets, int64_t *routing_nets);
/* Route record of routing net `net` (phase 1 or its latest reroute). */
int igr_router_route(igr_router *r, int net, int32_t *out, int cap, int *len);
/* Selected pins of design net `net` (net::init, src/database.hpp:38-243):
 * record npins, pins (file-layer positions, in the order net::init leaves
 * them: the iteration order of its robin_hood sets), nextra, extra pairs.
 * Available right after igr_router_open (no GPU needed). */
int igr_router_pins(igr_router *r, int net, int32_t *out, int cap, int *len);
/* Device demand of the grid ([l][x][y], routing layers). */
int igr_router_demand(igr_router *r, float *out);
void igr_router_close(igr_router *r);

/* Synthetic ISPD2024-style design (no counterpart in InstantGR, whose
 * benchmarks are external).  cfg: 0..4 = the configurations of the
 * benchmark suite of this project; scale (0,1] shrinks the net count. */
int igr_generate(int cfg, uint64_t seed, double scale, const char *cap_path, const char *net_path);
/* Same, with explicit sizes. */
int igr_generate_custom(int X, int Y, int nets, uint64_t seed, int cap_mode, double block_frac, int pin_mode,
                        double hifanout_frac, double bbox_median, double bbox_sigma, int hotspots,
                        double hotspot_frac, const char *cap_path, const char *net_path);

/* ------------------------------------------------------------------ device operators */

typedef struct igr_grid_desc {
    int32_t L, X, Y;            /* routing layers (9), grid */
    int32_t dir0;               /* direction of routing layer 0: 0 = horizontal, 1 = vertical */
    const int32_t *x_edge_len;  /* [X-1] */
    const int32_t *y_edge_len;  /* [Y-1] */
    double unit_wire, unit_via;
    const double *short_cost;   /* [L] overflow weight per routing layer */
    const float *capacity;      /* [L][X][Y] */
} igr_grid_desc;

/* Device state of one grid: capacity, demand, cost tables, difference array,
 * timestamps (build_cuda_database, src/database_cuda.hpp:2096-2362). */
int igr_create(const igr_grid_desc *g, igr_ctx **out);
int igr_destroy(igr_ctx *c);
const char *igr_last_error(const igr_ctx *c);

/* Test hooks (no counterpart in InstantGR, whose failures end the process):
 * process-wide settings that let tests reach paths the default sizes do not,
 * and make the device's bounded waits run out without faulting anything.
 * Every setting applies to launches made after the call, from any context.
 *   IGR_HOOK_RESET            every hook back to its default (value ignored)
 *   IGR_HOOK_WAIT_NS          limit of every grid-barrier and tensor-core
 *                             mbarrier wait in ns (default 2e9); a wait that
 *                             runs out sets IGR_ERR_TIMEOUT, the kernel drains
 *                             its own work in flight and returns
 *   IGR_HOOK_BARRIER_PHANTOM  arrivals the colouring's grid barriers wait for
 *                             that never come (default 0): its first barrier
 *                             then runs out by construction
 *   IGR_HOOK_MBAR_PROBE       1: every seed-network GEMM first waits on an
 *                             mbarrier phase that nothing completes, before it
 *                             issues any MMA (default 0)
 *   IGR_HOOK_COLOR_KEEP_MAP   igr_color_batches keeps the round-0 claim map up
 *                             to date across batches (1, default) or clears
 *                             and re-claims it every batch (0); the batches
 *                             are the same
 *   IGR_HOOK_DAG_SPLIT_NETS   DAG batches of at least this many nets (default
 *                             4096) run their DAGs of at most 64 nodes in
 *                             2-warp CTAs beside the larger ones on a second
 *                             stream; the routes are the same
 *   IGR_HOOK_COLOR_KEEP_MIN_NETS  the router keeps the round-0 claim map up
 *                             to date in colourings of at least this many nets
 *                             (default 2,000,000); the batches are the same
 *   IGR_HOOK_SHAPE_DEDUPE     the router keeps each conflict point and each
 *                             claimed cell of a net once (1, default) or
 *                             every repetition (0); the batches are the same
 *   IGR_HOOK_DAG_STAGE_NODES  the DAG DP keeps the DAG of a net of at most
 *                             this many nodes (0..4096, default 1024; 0: none)
 *                             in shared memory while it routes it, where it
 *                             fits; the routes are the same */
enum {
    IGR_HOOK_RESET = 0,
    IGR_HOOK_WAIT_NS = 1,
    IGR_HOOK_BARRIER_PHANTOM = 2,
    IGR_HOOK_MBAR_PROBE = 3,
    IGR_HOOK_COLOR_KEEP_MAP = 4,
    IGR_HOOK_DAG_SPLIT_NETS = 5,
    IGR_HOOK_COLOR_KEEP_MIN_NETS = 6,
    IGR_HOOK_SHAPE_DEDUPE = 7,
    IGR_HOOK_DAG_STAGE_NODES = 8,
};
int igr_test_hook(int key, int64_t value);

/* Demand in and out ([l][x][y]).  Setting demand marks every track dirty. */
int igr_set_demand(igr_ctx *c, const float *demand);
int igr_get_demand(igr_ctx *c, float *demand);
/* Timestamps and the difference array ([l][x][y]), for replay and checks. */
int igr_get_stamp(igr_ctx *c, int32_t *stamp);
int igr_get_pre(igr_ctx *c, int32_t *pre);

/* Fused cost refresh: wire cost, via cost and per-track prefix sums
 * (update_wcost_cuda_ispd24 + update_vcost_ispd24 + compute_presum,
 * src/graph.hpp:40-71, :101-104, :405-430).  only_dirty != 0 recomputes only
 * tracks whose demand changed since the previous refresh. */
int igr_cost_refresh(igr_ctx *c, int only_dirty);
/* Cost tables after a refresh: vcost f32 and presum f64, [l][x][y]. */
int igr_get_costs(igr_ctx *c, float *vcost, double *presum);
/* Loads a cost map (for replaying a reference cost map into the DP). */
int igr_set_costs(igr_ctx *c, const float *vcost, const double *presum);
/* Grid state to a file and back, for parity checks and replay: the file holds
 * "IGRSTAT1", int32 L, X, Y, then demand (f32), vcost (f32), presum (f64),
 * stamp (i32) and the wire difference array (i32), each [l][x][y], in the
 * host's byte order.  Loading needs a context of the same L, X, Y
 * (IGR_ERR_INVALID otherwise; IGR_ERR_IO / IGR_ERR_FORMAT for an unreadable
 * or short file); the loaded costs count as fresh and every track as holding
 * a pending wire commit.  Replaces the dump hooks planned for the reference
 * (the survey's replay patch); InstantGR itself has none. */
int igr_dump_state(igr_ctx *c, const char *path);
int igr_load_state(igr_ctx *c, const char *path);

/* Phase-1 tree DP (Lshape_route_cuda, src/Lshape_route.hpp:9-153) for a
 * batch of n nets.  Trees: nodes in DFS preorder (node_off[n+1] CSR), node
 * positions in InstantGR's encoding with layer 9 for Steiner nodes, par[i] the
 * local index of the parent (-1 at the root).  route_cap[k] ints are
 * available for net k; routes are written to routes_out at route_off[k].
 * Wires go to the difference array; call igr_commit_wires afterwards. */
int igr_pattern_route(igr_ctx *c, int n, const int32_t *node_off, const int32_t *nodes, const int32_t *par,
                      const int64_t *route_off, const int32_t *route_cap, int32_t *routes_out, int32_t stamp);

/* The same tree DP for callers that cannot let a library allocate device
 * memory: hosts that give the whole GPU to their own pool allocator, loops
 * that cannot afford the device-wide synchronisation a cudaMalloc may cause,
 * and processes that must fix their footprint before they start.  It has no
 * counterpart in InstantGR.
 *
 * Every pointer is DEVICE memory owned by the caller: node_off[n+1],
 * nodes/par[total_nodes], route_off/route_cap[n], routes[routes_len].  Inputs
 * must be complete on the device when the call starts; the call runs on the
 * context's stream and returns when the routes and the difference array are
 * written (then call igr_commit_wires as usual).  Results are identical to
 * igr_pattern_route's.
 *
 * The DP's scratch (layer tables of nets with more than 16 tree nodes, 504
 * bytes per such node, plus 12 bytes per net and a work counter: room for
 * about 133,000 such nodes in a small call and about 108,000 at
 * IGR_STATIC_MAX_NETS nets) lives in one
 * fixed array of IGR_STATIC_SCRATCH_BYTES in the library's device image, held
 * by every GPU that loads the library until the process exits.  A call with
 * more than IGR_STATIC_MAX_NETS nets, or whose large nets need more scratch
 * than the array holds, returns IGR_ERR_CAPACITY and runs nothing.  The call
 * allocates no device memory; its first call on a device looks up the
 * array's device address, so make that first call before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (from several
 * threads or contexts of one device) race on it, so serialise them. */
#define IGR_STATIC_SCRATCH_BYTES (64u << 20)
#define IGR_STATIC_MAX_NETS (1 << 20)
int igr_pattern_route_static(igr_ctx *c, int n, const int32_t *node_off, int64_t total_nodes, const int32_t *nodes,
                             const int32_t *par, const int64_t *route_off, const int32_t *route_cap, int32_t *routes,
                             int64_t routes_len, int32_t stamp);
/* Difference-array commit (compute_presum_general + commit_all_edge + memset,
 * src/graph.hpp:74-137). */
int igr_commit_wires(igr_ctx *c, int32_t stamp);
/* Via demand of n route records (commit_via_demand, src/graph.hpp:496-543),
 * K = +1 to add, -1 to remove. */
int igr_commit_vias(igr_ctx *c, int n, const int64_t *route_off, const int32_t *routes, int32_t stamp, int32_t K);
/* Wire demand of n route records by atomics (commit_wire_demand,
 * src/graph.hpp:468-495), K = -1 for rip-up. */
int igr_ripup_wires(igr_ctx *c, int n, const int64_t *route_off, const int32_t *routes, int32_t stamp, int32_t K);
/* Rip-up marking (mark_overflow_edges/_nets, src/graph.hpp:432-466). */
int igr_mark_overflow(igr_ctx *c, int n, const int64_t *route_off, const int32_t *routes, int32_t threshold,
                      int32_t min_edges, uint8_t *is_of_out);
/* Congestion view (extract_congestionView*, src/graph.hpp:545-584), [x][y]. */
int igr_congestion_view(igr_ctx *c, float *xsum, float *ysum);
/* Overflow cost and counters (report_score, src/graph.hpp:148-169). */
int igr_score(igr_ctx *c, double *wirelength, double *vias, double *overflow);

/* Batch colouring (generate_batches_rsmt_gpu, src/database_cuda.hpp:437-631),
 * deterministic.  Nets in priority order (the last wins conflicts); CSR of
 * 2-D conflict points and of tree segments (pairs of 2-D cells). */
int igr_color_batches(igr_ctx *c, int n, const int32_t *pt_off, const int32_t *pts, const int32_t *h_off,
                      const int32_t *hseg, const int32_t *v_off, const int32_t *vseg, int32_t sparsity,
                      int32_t *batch_out, int32_t *n_batches);

/* Phase-2 DAG DP (precompute_cost_edge + Lshape_route_node_layer_change_cuda
 * + get_routing_tree_layer_change_cuda, src/Lshape_route_detour.hpp:123-195,
 * :281-406, :520-694) for a batch of n nets.  DAG CSR per net: nodes in
 * topological order (children before parents is NOT required; depth[] gives
 * the level), par_off/par/child_slot per node, child_num per node. */
int igr_dag_route(igr_ctx *c, int n, const int32_t *node_off, const int32_t *nodes, const int32_t *depth,
                  const int32_t *par_off, const int32_t *par, const int32_t *child_slot, const int32_t *child_num,
                  const int64_t *route_off, const int32_t *route_cap, int32_t *routes_out, int32_t stamp);

/* ------------------------------------------------------------------ host passes */

/* Detour DAG of one net (net::generate_detours_reconstruct,
 * src/database_cuda.hpp:1429-2086).  Tree of ntree nodes: positions pos[]
 * (layer 9 marks Steiner nodes), adjacency CSR adj_off[ntree+1]/adj.
 * Congestion view xsum/ysum as returned by igr_congestion_view.  The result
 * record is m, nodes[m], par_num[m], child_num[m], depth[m], E, par[E],
 * child_idx[E], npoints, points[npoints] with nodes in topological order
 * (parents first).  *len receives its length; nothing is written when
 * cap < *len. */
int igr_build_dag(int X, int Y, int mode, int ntree, const int32_t *pos, const int32_t *adj_off, const int32_t *adj,
                  const float *xsum, const float *ysum, int32_t *out, int64_t cap, int64_t *len);

/* Detour DAGs of n trees built on the device, one thread per tree (the
 * construction of igr_build_dag, which it replaces for the rip-up passes of
 * the router: Lshape_route_detour.hpp:702-748 calls
 * net::generate_detours_reconstruct, src/database_cuda.hpp:1429-2086, per
 * net on host threads).  Tree k: nodes tree_off[k] .. tree_off[k+1]-1 of
 * pos[]; node v's neighbours adj[adj_off[v] .. adj_off[v+1]) as indices
 * local to its tree (adj_off has tree_off[n] + 1 entries).  The records, in
 * igr_build_dag's format, are written end to end to out; rec_off[n+1]
 * receives their offsets and *len the total length; nothing is written to
 * out when cap < *len.  Needs a GPU. */
int igr_build_dags(int X, int Y, int mode, int n, const int32_t *tree_off, const int32_t *pos,
                   const int32_t *adj_off, const int32_t *adj, const float *xsum, const float *ysum, int32_t *out,
                   int64_t cap, int64_t *rec_off, int64_t *len);

/* Steiner provider used in place of FLUTE (flute::flute, src/flute.hpp:1239;
 * its POST9.dat table is absent).  Nodes: distinct input points in ascending
 * (x, y) order, then Steiner points; edges as node index pairs. */
int igr_steiner(int n, const int32_t *x, const int32_t *y, int32_t *node_x, int32_t *node_y, int cap_nodes,
                int *n_nodes, int32_t *edges, int cap_edges, int *n_edges);

/* ------------------------------------------------------------------ learned congestion seed
 *
 * A BF16 convolutional encoder-decoder (six 3x3 convolutions, 32-64
 * channels, FP32 accumulation in TMEM on the tcgen05 tensor cores) that
 * predicts the routed demand of every layer from placement features, run on
 * 256 x 256 GCell tiles with a 16-GCell halo.  No counterpart in InstantGR;
 * the router uses a model attached with igr_router_set_seed.  Maps are
 * channels-last [X][Y][16] float arrays: features = pins, RUDY-H, RUDY-V,
 * blocked-layer fraction, capacity of file layers 0..9 (scaled by 1/8), 0, 0;
 * predictions/targets = demand of file layers 0..9 (scaled by 1/8), 0 x 6. */
typedef struct igr_seed igr_seed;
int igr_seed_create(uint64_t init_seed, igr_seed **out);  /* He-normal initialisation */
int igr_seed_destroy(igr_seed *m);
const char *igr_seed_last_error(const igr_seed *m);
/* Tile size with halo (even) and halo; default 288 and 16. */
int igr_seed_set_tile(igr_seed *m, int size, int halo);
/* All parameters (per layer: weights [cout][3][3][cin], then biases); *n gets the count. */
int igr_seed_params(igr_seed *m, float *out, int64_t cap, int64_t *n);
int igr_seed_set_params(igr_seed *m, const float *params, int64_t n);
/* Features of an opened router's design ([X][Y][16]), on the host threads. */
int igr_seed_features(igr_router *r, float *out);
/* The same features computed on the device from the router's resident trees,
 * as a seeded run computes them (brings up the device state when needed); the
 * RUDY channels are summed in fixed point there and agree with
 * igr_seed_features to the BF16 rounding. */
int igr_seed_features_device(igr_router *r, float *out);
/* Training maps kept in device memory: explicit maps, or the features and the
 * routed demand of a router's last run. */
int igr_seed_add_map(igr_seed *m, int X, int Y, const float *features, const float *target, int32_t *map_id);
int igr_seed_add_routed(igr_seed *m, igr_router *r, int32_t *map_id);
/* `steps` Adam steps on batches of `tiles` random tiles of training maps
 * 0..nmaps-1 (0: all); loss_curve[steps] (optional) receives the mean squared
 * error of each step. */
int igr_seed_train(igr_seed *m, int steps, int tiles, float lr, uint64_t seed, int nmaps, double *loss_curve);
/* Errors of the prediction of stored map `map`: out[0] mean squared error,
 * [1] mean absolute error, [2] MAE of predicting zero, [3] MAE of predicting
 * each layer's mean demand over the map. */
int igr_seed_eval(igr_seed *m, int map, double *out, int n);
/* Prediction of a whole feature map (tiled). */
int igr_seed_predict(igr_seed *m, int X, int Y, const float *features, float *pred);
/* Device time of the network's forward convolutions (the tcgen05 implicit
 * GEMMs) over `tiles` tiles of the current tile size, averaged over `reps`
 * passes after one untimed pass: layer_ms[i] = milliseconds of convolution i
 * per pass (CUDA events on the model's stream), layer_flops[i] = its
 * multiply-add FLOPs per pass (2 x output pixels x 9 x cin x cout); both
 * arrays hold IGR_SEED_CONVS entries.  The tiles hold the last inputs loaded
 * (zeros at first): the time does not depend on the values. */
#define IGR_SEED_CONVS 6
int igr_seed_time_forward(igr_seed *m, int tiles, int reps, double *layer_ms, double *layer_flops);
/* Attaches a model to a router (mode 0: none, 1: every run seeded, 2: a seeded
 * run and a plain run, the better total score kept).  Seeding adds alpha x the
 * predicted demand (kind 0) or alpha x the predicted overflow over capacity
 * (kind 1), rounded to half units, to the demand during phase 1 and removes
 * it after; with levels > 0 the seed shrinks in that many steps as the
 * phase-1 batches commit.  kind + 2 (2: demand, 3: overflow) also orders
 * rip-up-and-reroute by predicted overflow (nets of higher predicted overflow
 * first) instead of InstantGR's HPWL order; that order makes the reroute
 * colourings take more rounds (800k-net design: 1.05x plain's time in the
 * HPWL order, 0.72x with it).  The model must outlive the router's runs. */
int igr_router_set_seed(igr_router *r, igr_seed *m, double alpha, int mode, int kind, int levels);
/* Seed statistics of the last run: [0] 1 if the seeded result was kept (mode 2),
 * [1] seeded total score, [2] plain total score (mode 2), [3] prediction ms.
 * Scores are the evaluator's totals (igr_router_evaluate); after a mode-1 run
 * the seeded score is computed by the first call. */
int igr_router_seed_stats(igr_router *r, double *out, int n);
/* One forward and backward pass on T tiles (x, target: [T][size][size][16])
 * without an update: loss and the gradient of every parameter (layout of
 * igr_seed_params), for gradient checks. */
int igr_seed_grad(igr_seed *m, int T, const float *x, const float *target, double *loss, float *grads);

#ifdef __cplusplus
}
#endif

#endif /* INSTANTGR_B200_H */
