/*
 * CPU oracle for the routing hot path — TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatements of InstantGR's device kernels, in the reference's own
 * data layout ([l][x][y], 81-entry DP tables, one net at a time), used by the
 * tests, the smoke check and the CPU baseline of the benchmark as the checker.
 * Nothing in the product links or calls this code.
 *
 * Parity is pinned against golden vectors produced by the reference itself
 * (its kernels driven by oracle/ref_harness.cu, its host front end by
 * oracle/ref_front.cu); see tests/golden/.
 *
 * One deliberate difference: the reference evaluates the overflow cost with
 * the CUDA intrinsic __expf; the oracle uses the C library exp() in double
 * precision, so cost tables agree within a relative tolerance (1e-5), not
 * bit for bit.  The DP and commit restatements take the cost map as input, so
 * their integer outputs are compared exactly.
 */
#ifndef IGR_ORACLE_H
#define IGR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    int L, X, Y, DIR;       /* routing layers, grid, direction of routing layer 0 */
    const int *xlen, *ylen; /* [X-1], [Y-1] */
    double unit_wire, unit_via;
    const double *short_cost; /* [L] */
    const float *cap;         /* [L][X][Y] */
} orc_grid;

/* update_wcost_cuda_ispd24 + update_vcost_ispd24 + compute_presum
 * (src/graph.hpp:40-71, :101-104, :405-430); outputs in [l][x][y]. */
void orc_cost_refresh(const orc_grid *g, const float *demand, float *wcost, float *vcost, double *presum);

/* Lshape_route_cuda (src/Lshape_route.hpp:9-153) for n nets, sequentially.
 * pre (difference array) and stamp are updated in place; routes written at
 * route_off[k]. Returns 0, or -1 if a route record overflowed its capacity. */
int orc_pattern_route(const orc_grid *g, const float *vcost, const double *presum, int n, const int *node_off,
                      const int *nodes, const int *par, const int64_t *route_off, const int *route_cap, int *routes,
                      int *pre, int *stamp_arr, int stamp);

/* compute_presum_general + commit_all_edge + memset (src/graph.hpp:74-137).
 * Returns the wirelength added. */
int64_t orc_commit_wires(const orc_grid *g, int *pre, float *demand, int *stamp_arr, int stamp);

/* commit_via_demand (src/graph.hpp:496-543). Returns the via count added. */
int64_t orc_commit_vias(const orc_grid *g, int n, const int64_t *route_off, const int *routes, float *demand,
                        const int *stamp_arr, int stamp, int K);

/* commit_wire_demand (src/graph.hpp:468-495). Returns the wirelength added. */
int64_t orc_ripup_wires(const orc_grid *g, int n, const int64_t *route_off, const int *routes, float *demand,
                        int *stamp_arr, int stamp, int K);

/* mark_overflow_edges + compute_presum_general + mark_overflow_nets
 * (src/graph.hpp:432-466). */
void orc_mark_overflow(const orc_grid *g, const float *demand, int n, const int64_t *route_off, const int *routes,
                       int threshold, int min_edges, uint8_t *is_of);

/* extract_congestionView{,_xsum,_ysum} (src/graph.hpp:545-584), [x][y]. */
void orc_congestion_view(const orc_grid *g, const float *demand, float *xsum, float *ysum);

/* Overflow cost of add_all_overflow_cost (src/graph.hpp:148-157), exp() in double. */
double orc_overflow_cost(const orc_grid *g, const float *demand);

/* Batch colouring with the phase semantics of generate_batches_rsmt_gpu
 * (src/database_cuda.hpp:288-631) made deterministic: claim, commit, block and
 * release as separate phases.  Returns the number of batches. */
int orc_color(int X, int Y, int n, const int *pt_off, const int *pts, const int *h_off, const int *hseg,
              const int *v_off, const int *vseg, int sparsity, int *batch);

/* Phase-2 DAG routing (src/Lshape_route_detour.hpp:123-195, :281-406,
 * :520-694) of one batch; node indices are batch-global.  Routes are emitted
 * per node in node order.  Returns 0, or -1 on a record overflow. */
int orc_dag_route(const orc_grid *g, const float *vcost, const double *presum, int n, const int *node_off,
                  const int *nodes, const int *depth, const int *par_off, const int *par, const int *child_slot,
                  const int *child_num, const int64_t *route_off, const int *route_cap, int *routes, int *pre,
                  int *stamp_arr, int stamp);

#ifdef __cplusplus
}
#endif
#endif
