/*
 * grb_oracle.h -- CPU restatement of GRotor's routing hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * grotor_b200/: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference leg of bench.py may load it.  The product never links it and
 * has no CPU fallback.
 *
 * Every function restates the reference's algorithm from its source (file:line
 * cited at each definition, paths relative to the GRotor project root).  Cost
 * values use the host's expf where the reference uses CUDA's __expf, so costs
 * agree with the GPU within 1e-6 relative -- or bit for bit once a table of
 * the device's own exponential values is installed (orc_set_exp_table); every
 * other step (prefix addition order, DP comparisons, tie-breaks, demand,
 * batching) is exact.  Parity of the
 * restatement is pinned against outputs of the reference itself (see
 * tests/golden/ and oracle/ref_harness.cu).
 *
 * Grid layout: IDX(l,x,y) = (l*X + x)*Y + y; layer l carries wires along y when
 * ((l & 1) ^ DIR) is 1, along x otherwise (router_state.hpp:267,
 * full_update.cuh:43).  Demand is kept in int32 half-units (a wire edge adds 2,
 * a split via landing adds 1), which is exact and converts to the reference's
 * float demand bit-for-bit (demand = half * 0.5f).
 */
#ifndef GRB_ORACLE_H
#define GRB_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    int32_t L, X, Y, DIR;
    double unit_wire, unit_via, of_cost_scale;
    const double* short_costs;   /* [L] overflow weight per routing layer */
    const int32_t* x_edge_len;   /* [X-1] */
    const int32_t* y_edge_len;   /* [Y-1] */
    const float* capacity;       /* [L*X*Y] */
    int32_t integer_wire;        /* 1: GGR build's wire costs, clamped to [0, 1e7] and truncated (full_update.cuh:47-50) */
} orc_grid;

/* The cost model's exponential (full_update.cuh:9-14).  By default the host's
 * expf stands in for the device's __expf, which agrees within 1e-6 relative.
 * orc_exp_args writes, ascending and without repeats, every argument the cost
 * model can pass to the exponential on this grid for cell demands of 0 ..
 * max_demand_half half-units (at most `cap` of them; returns the count).
 * orc_set_exp_table installs the device's values y[i] = exp(x[i]) for such
 * arguments (n = 0 removes the table); with it every cost value equals the
 * device's bit for bit.  Arguments missing from an installed table use expf
 * and are counted by orc_exp_table_misses (reset by orc_set_exp_table). */
int64_t orc_exp_args(const orc_grid* g, int32_t max_demand_half, float* out, int64_t cap);
void orc_set_exp_table(int64_t n, const float* x, const float* y);
int64_t orc_exp_table_misses(void);

/* Full cost recompute: wcost/vcost from capacity and demand. */
void orc_cost_full(const orc_grid* g, const int32_t* demand_half, float* wcost, float* vcost);

/* Per-track double prefix of wcost in the reference's addition order. */
void orc_presum(const orc_grid* g, const float* wcost, double* presum);

/* Same prefix computed by the literal log-step (Sklansky) loop of the full scan;
 * used by the tests to prove orc_presum's single-pass form adds in the same order. */
void orc_presum_logstep(const orc_grid* g, const float* wcost, double* presum);

/* L-shape tree DP for the nets of one batch (thread-per-net semantics).
 * node_off is the CSR over all nets of the plan (global); nets are ids[0..n).
 * Writes routes[route_off[id] ...] = [count, a0, b0, a1, b1, ...].
 * Returns 0, or -1-i if net i's output would exceed its route capacity. */
int orc_lshape_batch(const orc_grid* g, const float* vcost, const double* presum,
                     int32_t n, const int32_t* ids, const int32_t* node_off,
                     const int32_t* nodes, const int32_t* parents,
                     const int64_t* route_off, int32_t* routes);

/* Wire then via demand commit of one batch (K = +1 commit, -1 rip-up). */
void orc_commit_batch(const orc_grid* g, int32_t n, const int32_t* ids,
                      const int64_t* route_off, const int32_t* routes,
                      int32_t stamp, int32_t K, int32_t* demand_half, int32_t* timestamp,
                      double* total_wirelength, int64_t* total_vias);

/* Exact greedy first-fit batching.  order[0..n) are net ids; geometry CSRs are
 * indexed by net id.  Writes batch_of[i] for order position i and returns the
 * number of batches. */
int32_t orc_batches(int32_t X, int32_t Y, int32_t n, const int32_t* order,
                    const int32_t* point_off, const int32_t* points,
                    const int32_t* hseg_off, const int32_t* hsegs,
                    const int32_t* vseg_off, const int32_t* vsegs,
                    int32_t limit, int32_t sparsity, int32_t* batch_of);

/* Rip-up classification: is_of[id] = route of net crosses > 10 overflowed edges
 * (demand >= capacity + threshold). routes_of_net: route_off per net id. */
void orc_ripup_classify(const orc_grid* g, const int32_t* demand_half, int32_t threshold,
                        int32_t n_nets, const int64_t* route_off, const int32_t* routes,
                        uint8_t* is_of);

/* Congestion view: worst (demand - capacity) over layers per (x,y), flag and
 * row/column float prefix sums. */
void orc_congestion_view(const orc_grid* g, const int32_t* demand_half,
                         uint8_t* congestion, float* xsum, float* ysum);

/* Whole L-shape stage over an explicit batch plan: for each batch, ++stamp,
 * full cost refresh, DP, commit.  ids/batch_off describe the plan in execution
 * order.  nthreads > 1 solves the nets of a batch on that many host threads
 * (results are independent of the thread count). */
int orc_lshape_stage(const orc_grid* g, int32_t n_batches, const int32_t* batch_off,
                     const int32_t* ids, const int32_t* node_off, const int32_t* nodes,
                     const int32_t* parents, const int64_t* route_off, int32_t* routes,
                     int32_t* demand_half, int32_t* timestamp, int32_t* stamp,
                     double* total_wirelength, int64_t* total_vias, int32_t nthreads);

/* FLT DAGs of a stage's nets, CSR by net id (nets outside the stage have empty
 * ranges).  Per node: 3-D coordinate (layer 9 marks a node with no pin layer),
 * depth, child-slot count, cumulative parent-edge count within the net.  Per
 * edge, grouped by child node: parent node (net-local) and source slot
 * child * 10 + slot index at the parent (flt_topology.hpp:15-16, 52-70). */
typedef struct orc_flt {
    const int32_t* node_off;
    const int32_t* coord;
    const int32_t* depth;
    const int32_t* children;
    const int32_t* parent_end;
    const int32_t* edge_off;
    const int32_t* edge_parent;
    const int32_t* edge_slot;
} orc_flt;

/* FLT stage (flt.cuh:141-168) over an explicit batch plan in execution order:
 * per batch, optionally remove the nets' phase-one routes (K = -1, own stamp),
 * ++stamp, full cost refresh, mid-edge layer-change tables, bottom-up solve,
 * top-down trace into the phase-two routes (routes2 at route2_off[id], count
 * word first), commit of the phase-two routes.  Returns 0, or 3 when a net's
 * route storage overflows, or 4 for an unroutable net. */
int orc_flt_stage(const orc_grid* g, const orc_flt* dags, int32_t n_batches, const int32_t* batch_off,
                  const int32_t* ids, const int64_t* route_off, const int32_t* routes,
                  const int64_t* route2_off, int32_t* routes2, int32_t remove_phase_one,
                  int32_t* demand_half, int32_t* timestamp, int32_t* stamp,
                  double* total_wirelength, int64_t* total_vias, int32_t nthreads);

/* Z-shape trees in the reference's encoding (zshape::encode_batch,
 * zshape_topology.hpp:59-121), CSR by net id: nodes in preorder from the
 * first leaf, 3-D coordinate (layer L = Steiner point) and up to three child
 * preorder indices per node (-1 = none). */
typedef struct orc_ztrees {
    const int32_t* node_off;
    const int32_t* coord;
    const int32_t* child;   /* [3 per node] */
} orc_ztrees;

/* Z-shape stage (pipeline_ggr.hpp:119-134) over an explicit batch plan in
 * execution order: per batch, full cost refresh, Z-shape DP and traceback per
 * net (zshape.cuh:42-388), conversion to route words (zshape_topology.hpp:
 * 249-290) at route_off[id], ++stamp, thread-per-net wire then via commit
 * (demand.cuh:129-232).  Returns the reference's status: 0, 1 (route storage),
 * 2 (no finite route), 3 (segment outside the grid). */
int orc_zshape_stage(const orc_grid* g, const orc_ztrees* trees, int32_t n_batches, const int32_t* batch_off,
                     const int32_t* ids, const int64_t* route_off, int32_t* routes, int32_t* demand_half,
                     int32_t* timestamp, int32_t* stamp, double* total_wirelength, int64_t* total_vias);

/* Bounding-box refinement of one first-fit group (zshape::generate_bbox_batches,
 * zshape_topology.hpp:7-57): nets sorted by box area (descending, larger id
 * first on ties), greedy rounds of at most max_batch nets with disjoint boxes.
 * bbox is [minx, maxx, miny, maxy] per net id.  Writes the refined batches
 * (ids, off) and returns their number. */
int32_t orc_bbox_batches(int32_t X, int32_t Y, int32_t n, const int32_t* group, const int32_t* bbox,
                         int32_t max_batch, int32_t* ids, int32_t* off);

/* Topology of every net from its Steiner tree: the batching geometry of
 * net::construct_rsmt (preprocess.hpp:95-123: the nodes' 2-D cells, then per
 * tree edge (i, j < i) in adjacency order two corner or end points and its
 * h / v segments) and the depth-first flattening of Lshape_route
 * (lshape.cuh:85-98: preorder from node 0, neighbours in adjacency order,
 * parent's preorder index).  pos: layer*X*Y + x*Y + y per node (layer L =
 * Steiner point); adj_off/adj: each node's neighbours (net-local indices).
 * Output buffers hold at most node_off[n] nodes, 3*node_off[n] points and
 * 2*node_off[n] segments of each kind; totals[0..2] receive the point, h- and
 * v-segment counts.  Returns 0, or -(net+1) for a net whose adjacency is not
 * a tree on its nodes. */
int orc_build_topology(int32_t X, int32_t Y, int32_t n, const int32_t* node_off, const int32_t* pos,
                       const int32_t* adj_off, const int32_t* adj, int32_t* nodes, int32_t* parents,
                       int32_t* point_off, int32_t* points, int32_t* hseg_off, int32_t* hsegs,
                       int32_t* vseg_off, int32_t* vsegs, int64_t* totals);

#ifdef __cplusplus
}
#endif
#endif
