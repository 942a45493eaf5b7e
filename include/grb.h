/*
 * grb.h -- C ABI of grotor_b200: GRotor's routing hot path on NVIDIA B200.
 *
 * The reference router (GRotor) has no plugin or FFI layer; its hot path sits
 * behind a handful of C++ functions called from its stage drivers.  Each entry
 * point below replaces one of them (reference file:line, paths relative to the
 * GRotor project root).  The host pipeline (CAP/NET parsing, net splitting,
 * RSMT/FLT topology construction, .out writer) stays in the caller.
 *
 * Conventions
 *  - Grid cell index IDX(l,x,y) = (l*X + x)*Y + y over the L routing layers
 *    (router_state.hpp:267).  Layer l carries wires along y when
 *    ((l & 1) ^ DIR) == 1, along x otherwise (DIR = direction of CAP layer 1,
 *    preprocess.hpp:1616).
 *  - Tree nodes are 3-D cell ids; Steiner nodes use layer L (preprocess.hpp:131).
 *  - Route words per net: [count, a0, b0, a1, b1, ...] where count is one past
 *    the last used word, exactly the reference's route record
 *    (lshape_warp.cuh:215-240); a pair with equal layers is a wire, otherwise a
 *    via stack.
 *  - Demand is int32 half-units (wire edge +2, split via landing +1 each side);
 *    demand_half * 0.5f equals the reference's float demand bit-for-bit.
 *  - Every call returns GRB_OK or an error code and never throws; the text of
 *    the last error is available from grb_last_error().  A context owns all of
 *    its device memory and one CUDA stream; it is not thread-safe.
 *  - There is no CPU fallback: every compute entry point runs CUDA kernels.
 */
#ifndef GRB_H
#define GRB_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRB_OK 0
#define GRB_EINVAL 1     /* bad argument or inconsistent input */
#define GRB_ENOMEM 2     /* device allocation failed */
#define GRB_ECUDA 3      /* CUDA runtime error */
#define GRB_ETIMEDOUT 4  /* a bounded device wait expired */
#define GRB_ELIMIT 5     /* route storage or batch-colour capacity exceeded */

#define GRB_MODE_PLAIN 0       /* one launch sequence per batch (reference structure) */
#define GRB_MODE_GRAPH 1       /* the plain sequence captured in one CUDA graph */
#define GRB_MODE_PERSISTENT 2  /* one cooperative kernel runs every batch */

typedef struct grb_ctx grb_ctx;

/* Routing grid and cost model: the device tables built by
 * build_cuda_database (preprocess.hpp:1625-1786). */
typedef struct grb_grid {
    int32_t L, X, Y, DIR;
    double unit_length_wire_cost;
    double unit_via_cost;
    double of_cost_scale;                   /* 1.0 on one GPU (router_state.hpp:37) */
    const double* unit_length_short_costs;  /* [L] overflow weight per routing layer */
    const int32_t* x_edge_len;              /* [X-1] */
    const int32_t* y_edge_len;              /* [Y-1] */
    const float* capacity;                  /* [L*X*Y] */
} grb_grid;

/* Per-net topology and batching geometry, indexed by net id (the reference's
 * net::rsmt DFS order, net::points, rsmt_h_segments, rsmt_v_segments;
 * lshape.cuh:85-103, preprocess.hpp:88-130). */
typedef struct grb_nets {
    int32_t n;
    const int32_t* node_off;   /* [n+1] */
    const int32_t* nodes;      /* DFS order, node 0 = root */
    const int32_t* parents;    /* parent index < child index, -1 at the root */
    const int64_t* route_off;  /* [n+1] word offsets; route capacity of net i = route_off[i+1]-route_off[i] */
    const int32_t* point_off;  /* [n+1] */
    const int32_t* points;     /* 2-D cell ids x*Y+y */
    const int32_t* hseg_off;   /* [n+1] */
    const int32_t* hsegs;      /* pairs (first, second), 2-D ids, step Y */
    const int32_t* vseg_off;   /* [n+1] */
    const int32_t* vsegs;      /* pairs (first, second), 2-D ids, step 1 */
} grb_nets;

typedef struct grb_stats {
    double total_wirelength;   /* RoutingStatistics::total_wirelength (router_state.hpp:17-20) */
    int64_t total_via_count;   /* RoutingStatistics::total_via_count */
    int32_t n_batches;
    int32_t stamp;             /* RouterState::global_timestamp after the call */
    double batching_ms;        /* device time of the last grb_plan_batches */
    double dag_ms;             /* device time of the last stage */
} grb_stats;

/* Start CUDA on `device` and load the library's stage kernels, so that a
 * caller can overlap this one-time cost with its input reading, as the
 * reference's main does with cudaFree(nullptr) and cudaFuncGetAttributes in
 * an asynchronous task while db::read and flute::readLUT run
 * (src/main.cu:101-106).  Optional: grb_create does the same when it has not
 * been called.  Safe to call from another thread than the context's. */
int grb_init_device(int32_t device);

/* Create a context on `device` and upload the grid (build_cuda_database,
 * preprocess.hpp:1625; initialize_incremental_cost, incremental_update.cuh:7). */
int grb_create(const grb_grid* grid, int32_t device, grb_ctx** out);
void grb_destroy(grb_ctx* ctx);
const char* grb_last_error(const grb_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for callers that time or order work. */
void* grb_stream(grb_ctx* ctx);

/* Zero demand, timestamps, statistics and routes; mark every cost dirty
 * (the state of a freshly built database; experiments/lshape_benchmark.cuh:86-99). */
int grb_reset(grb_ctx* ctx);

/* Upload per-net topology and geometry (host buffers; replaces the uploads in
 * Lshape_route, lshape.cuh:126-138, and the batching inputs). */
int grb_upload_nets(grb_ctx* ctx, const grb_nets* nets);

/* Every net's Steiner tree as FLUTE leaves it in net::rsmt after
 * construct_rsmt (preprocess.hpp:72-93 and 124-126): the node positions
 * (layer * X*Y + x*Y + y; layer L marks a Steiner point) and each node's
 * adjacency list (net-local node indices, in net::rsmt order). */
typedef struct grb_trees {
    int32_t n;
    const int32_t* node_off;   /* [n+1] */
    const int32_t* pos;        /* [node_off[n]] */
    const int32_t* adj_off;    /* [node_off[n]+1] offsets into adj */
    const int32_t* adj;        /* neighbours, net-local indices */
    const int64_t* route_off;  /* [n+1] as in grb_nets */
} grb_trees;

/* Topology construction on the device: from the trees, every net's DP tree
 * (the depth-first flattening of Lshape_route, lshape.cuh:85-98) and batching
 * geometry (net::points, rsmt_h_segments, rsmt_v_segments of construct_rsmt,
 * preprocess.hpp:95-123) are built on the GPU, in the same order as the
 * reference's host code; the context then holds the same nets as after
 * grb_upload_nets of the host-built arrays.  GRB_EINVAL if a net's adjacency
 * is not a tree on its nodes or a position is outside the grid. */
int grb_build_topology(grb_ctx* ctx, const grb_trees* trees);
/* Sizes of the context's net store: nodes, points, h-segments, v-segments. */
int grb_topology_sizes(grb_ctx* ctx, int64_t* sizes);
/* Copy the net store out (node_off, point_off, hseg_off, vseg_off: n+1
 * entries; segments as pairs); any pointer may be NULL. */
int grb_read_topology(grb_ctx* ctx, int32_t* node_off, int32_t* nodes, int32_t* parents, int32_t* point_off,
                      int32_t* points, int32_t* hseg_off, int32_t* hsegs, int32_t* vseg_off, int32_t* vsegs);

/* Exact first-fit batching of nets `order[0..n)` with at most `limit` nets per
 * batch (cudb::generate_batches_rsmt, generate_batches_cpu.hpp:7-73, and its
 * RT-core replacements).  The result becomes the context's plan in execution
 * order: batches reversed and flattened as in lshape.cuh:70-77.  If batch_of
 * is not NULL it receives the batch index of every order position. */
int grb_plan_batches(grb_ctx* ctx, const int32_t* order, int32_t n, int32_t limit, int32_t sparsity,
                     int32_t mode, int32_t* batch_of, int32_t* n_batches);

/* Set an explicit plan: net ids in execution order and batch offsets. */
int grb_set_plan(grb_ctx* ctx, const int32_t* ids, int32_t n, const int32_t* batch_off, int32_t n_batches);
/* Copy the current plan out (ids[n], batch_off[n_batches+1]). */
int grb_get_plan(grb_ctx* ctx, int32_t* ids, int32_t* batch_off, int32_t* n, int32_t* n_batches);

/* graph::refresh_cost (incremental_update.cuh:98-132): bring wcost, vcost
 * and the per-track prefix table up to date with demand. */
int grb_refresh_cost(grb_ctx* ctx);

/* Route batch `b` of the plan with L-shape patterns (Lshape_route_warp,
 * lshape_warp.cuh:105-247); writes routes only. */
int grb_route_batch(grb_ctx* ctx, int32_t b, int32_t stamp);

/* graph::commit_batch_demand (demand.cuh:313-319): K = +1 commits, K = -1
 * rips up the batch's routes. */
int grb_commit_batch(grb_ctx* ctx, int32_t b, int32_t stamp, int32_t K);

/* Run the whole L-shape stage over the plan: per batch ++stamp, refresh cost,
 * route, commit (Lshape_route::Lshape_route hot loop, lshape.cuh:153-179). */
int grb_lshape_stage(grb_ctx* ctx, int32_t mode, grb_stats* stats);

/* Rip-up classification (graph::ripup, congestion.cuh:114-136): is_of[id] = 1
 * for nets whose route crosses more than 10 edges with demand >= capacity +
 * threshold. */
int grb_ripup_classify(grb_ctx* ctx, int32_t threshold, uint8_t* is_of);

/* Allocation-free variant of grb_ripup_classify (no counterpart in the
 * reference).  Some callers cannot allocate device memory while they route:
 * processes that run under a fixed device-memory budget shared with another
 * framework's caching allocator, or steady-state loops that must not pay the
 * device-wide synchronisation cudaMalloc/cudaFree bring.  This entry point
 * allocates nothing: its scratch (one int per grid cell, one flag per net) is a
 * fixed array inside the library that every GPU loading the library holds until
 * the process exits: (4,194,304 + 262,144) ints = 17.0 MiB.  Limits: at most
 * 4,194,304 grid cells (L*X*Y) and 1,048,576 nets; larger designs get
 * GRB_ELIMIT.  The first call on a device looks up the array's device address
 * with that device current, so it should come before any stream capture; the
 * address is kept until the process exits, so a caller that resets the device
 * (cudaDeviceReset, which destroys the primary context) must not call this
 * entry point again in that process.  All calls share the one array (its
 * contents are those of the last call, and every word is rewritten before use),
 * so calls that overlap on the GPU -- two contexts or streams on the same
 * device at once -- race; serialise them.  Results equal grb_ripup_classify's. */
int grb_ripup_classify_noalloc(grb_ctx* ctx, int32_t threshold, uint8_t* is_of);

/* Autotuner (no counterpart in the reference).  Nets of every batch are
 * scheduled by size bucket (tree nodes <= 2, <= 8, <= 16, more; the
 * persistent form takes the largest bucket first).  what & 1 times the
 * per-batch DP launch of each bucket on the plan's largest batches for 1, 2,
 * 4 and 8 nets per CTA (arena sized to the bucket); what & 2 runs the
 * persistent stage from a reset state for candidate nets-per-grab sets of its
 * work queue (a nets-per-grab of 32 or more for the smallest bucket routes
 * those nets one per lane).  The choices stay in the context (and are copied to the
 * optional per_cta[4] / per_grab[4]).  Needs nets and a plan; leaves the
 * context reset (grb_reset).  Routes do not depend on the choices. */
int grb_autotune(grb_ctx* ctx, int32_t what, int32_t* per_cta, int32_t* per_grab);

/* ---- FLT stage (stage two of the default pipeline, flt.cuh:75-182) ------ */

/* Replace the batching geometry of the uploaded nets (net::points and
 * rsmt_h/v_segments after the FLT DAG builder has added its detour points,
 * preprocess.hpp:1002-1019) so that grb_plan_batches batches the FLT stage
 * (flt.cuh:92, limit 300000).  CSR by net id over the uploaded nets. */
int grb_upload_geometry(grb_ctx* ctx, const int32_t* point_off, const int32_t* points,
                        const int32_t* hseg_off, const int32_t* hsegs,
                        const int32_t* vseg_off, const int32_t* vsegs);

/* FLT DAGs of the stage's nets, CSR by net id over the uploaded nets (nets
 * outside the stage have empty ranges).  Exactly the reference's compact
 * topology (flt::Topology::emit, flt_topology.hpp:52-70; flt::Node/Edge,
 * :15-16): per node its 3-D coordinate (layer 9 = no pin layer), depth,
 * child-slot count and cumulative parent-edge count within the net; per edge,
 * grouped by child node, the parent (net-local) and the source slot
 * child * 10 + slot index at the parent.  route2_off gives each net's
 * phase-two route words (the reference reserves 100 per pin,
 * router_state.hpp:33, at pin_acc_num_phase2). */
typedef struct grb_flt_dags {
    const int32_t* node_off;     /* [n+1] */
    const int32_t* coord;
    const int32_t* depth;
    const int32_t* children;     /* <= 6 (flt_block.cuh:31-32) */
    const int32_t* parent_end;
    const int32_t* edge_off;     /* [n+1] */
    const int32_t* edge_parent;
    const int32_t* edge_source_slot;
    const int64_t* route2_off;   /* [n+1] */
} grb_flt_dags;

/* Upload FLT DAGs (host buffers; replaces flt::Workspace upload/assemble,
 * flt_workspace.cuh:156-224, and its CUB scan and depth sort).  Needs L == 9
 * routing layers (MAX_LAYER 10, flt_cost.cuh:14). */
int grb_upload_flt(grb_ctx* ctx, const grb_flt_dags* dags);

/* Run the FLT stage over the current plan (route_prepared_topology's batch
 * loop, flt.cuh:141-168): per batch, when remove_phase_one, remove the nets'
 * stage-one routes (commit with K = -1 under its own stamp), then ++stamp,
 * refresh_cost, layer-change tables (precompute_cost_edge), DAG solve and
 * trace (route_flt_block) into the phase-two routes, and commit of the
 * phase-two routes.  mode: GRB_MODE_PLAIN, GRAPH or PERSISTENT. */
int grb_flt_stage(grb_ctx* ctx, int32_t remove_phase_one, int32_t mode, grb_stats* stats);

/* Nets whose widest FLT DAG level holds more than `width` nodes are solved
 * and traced by a whole CTA (its threads over a level's nodes), the others by
 * one warp each; routes, demand and statistics are the same either way.
 * Default 32; a negative width routes every net with one warp. */
int grb_set_flt_block_width(grb_ctx* ctx, int32_t width);

/* ---- Maze stage of the CUGR2 pipeline (pipeline_cugr2.hpp:90-117) -------- */
/* maze::remove_routes (maze.cuh:24-64): remove the current routes of nets
 * ids[0..n) -- the phase-two words where phase2[k] is set, the stage-one
 * words otherwise -- from the demand and the statistics: each wire unit edge
 * -1, each via layer whose cell none of the net's own wires covers -1 at a
 * track end, else -1/2 on the two edges it lands between; the statistics
 * lose the net's edge lengths and via layers. */
int grb_remove_routes(grb_ctx* ctx, const int32_t* ids, int32_t n, const uint8_t* phase2);

/* graph::ripup's classification (congestion.cuh:8-58,114-136) on each net's
 * current route: the phase-two words for nets with phase2[id] set (the
 * reference's ripup_flag), the stage-one words otherwise. */
int grb_ripup_classify_phase2(grb_ctx* ctx, int32_t threshold, const uint8_t* phase2, uint8_t* is_of);

/* maze::routing_score (maze_quality.cuh:28-43): wirelength * unit wire cost +
 * vias * unit via cost + the overflow cost of every edge cell, reduced in a
 * fixed order (1024 blocks of 256 threads, a halving tree per block, the
 * partials in order), so equal states give equal scores bit for bit. */
int grb_routing_score(grb_ctx* ctx, double* score);

/* maze::Checkpoint (maze_quality.cuh:55-104), device part: grb_checkpoint
 * saves the demand and the statistics, grb_restore puts them back and
 * marks every cost for recomputation at the next refresh.  The route words
 * and rip-up flags are the caller's (the reference keeps them in host copies
 * too, pipeline_cugr2.hpp:14-61). */
int grb_checkpoint(grb_ctx* ctx);
int grb_restore(grb_ctx* ctx);

/* ---- .out writer (graph::output_nets, output.hpp:79-112) ---------------- */
/* Output records in output order, as graph::collect_output_nets hands them to
 * the writer (output.hpp:16-26): per record its name, its pins (3-D positions;
 * a pin on layer 0 is written as a via to layer 1), extra route pairs (3-D
 * positions, two per segment) and subnets (net ids of the context), each with
 * its rip-up flag (RouterState::ripup_flag_cpu: 1 selects the phase-two
 * routes). */
typedef struct grb_out_records {
    int32_t n;
    const int64_t* name_off;       /* [n+1] into names */
    const char* names;
    const int32_t* pin_off;        /* [n+1] */
    const int32_t* pins;
    const int32_t* extra_off;      /* [n+1] */
    const int32_t* extra;
    const int32_t* sub_off;        /* [n+1] */
    const int32_t* subnets;
    const uint8_t* sub_phase2;
} grb_out_records;

/* Receives the text in order; returns 0 to go on. */
typedef int (*grb_out_sink)(const char* data, int64_t bytes, void* user);

/* Format the records' .out text on the device -- exactly the bytes
 * graph::output_nets writes through grotor::RouteWriter (output_writer.hpp:
 * 29-43) from the context's current routes (stage one, and phase two for
 * flagged subnets) -- and leave it for grb_drain_out.  Returns its size in
 * *bytes.  The formatting is queued on the context's stream; the routes it
 * reads are those of the work queued before it. */
int grb_format_out(grb_ctx* ctx, const grb_out_records* records, int64_t* bytes);

/* Hand the formatted text to `sink` in order, in chunks of 64 MiB: chunk k+1
 * is copied (on the context's copy stream) while the sink consumes chunk k.
 * May run on another host thread while the calling thread queues further
 * stage work on the same context (the drain allocates nothing and touches no
 * other state); one text at a time: grb_format_out refuses while one is
 * pending. */
int grb_drain_out(grb_ctx* ctx, grb_out_sink sink, void* user);

/* Copy all phase-two route words (route2_off[n] words) to the host. */
int grb_read_routes2(grb_ctx* ctx, int32_t* routes2);
/* Replace all phase-two route words (route2_off[n] words of the last
 * grb_upload_flt) from the host: the routes of nets with phase-two storage
 * but no DAG in this stage, carried over from an earlier stage
 * (reserve_reroute_storage, pipeline_cugr2.hpp:14-63), or restored after a
 * rejected stage. */
int grb_write_routes2(grb_ctx* ctx, const int32_t* routes2);

/* ---- Z-shape stage (the reference's GGR pipeline, pipeline_ggr.hpp:8-144) */

/* Wire-cost mode of the cost tables: 0 = default; 1 = the GGR build's integer
 * wire costs, clamped to [0, 1e7] and truncated (full_update.cuh:47-50),
 * which the Z-shape stage's integer DP expects.  Takes effect at the next
 * cost refresh (every cell is recomputed). */
int grb_set_wire_cost_mode(grb_ctx* ctx, int32_t integer_wire);

/* Z-shape trees, CSR by net id over the uploaded nets, in the reference's
 * encoding (zshape::encode_batch, zshape_topology.hpp:59-121): nodes in
 * preorder from the tree's first leaf; per node its 3-D coordinate (layer L =
 * Steiner point) and up to three child preorder indices (-1 = none). */
typedef struct grb_zshape_trees {
    const int32_t* node_off;   /* [n+1] */
    const int32_t* coord;
    const int32_t* child;      /* [3 per node] */
} grb_zshape_trees;

/* Upload Z-shape trees (host buffers); also derives every net's bounding box
 * and allocates the DP planes (22 int planes of (L+1) * max(X,Y)^2). */
int grb_upload_zshape(grb_ctx* ctx, const grb_zshape_trees* trees);

/* Refine every batch of the current plan into bounding-box batches
 * (zshape::generate_bbox_batches, zshape_topology.hpp:7-57: box area
 * descending, rounds of at most max_batch nets with disjoint boxes) and make
 * the reversed list the plan (pipeline_ggr.hpp:51-55).  The current plan must
 * hold the first-fit groups in execution order (as grb_plan_batches leaves
 * it).  bbox: [minx, maxx, miny, maxy] per net id, or NULL for the boxes of
 * the uploaded Z-shape trees.  max_batch <= 256 (the reference uses 250). */
int grb_plan_bbox_batches(grb_ctx* ctx, const int32_t* bbox, int32_t max_batch, int32_t* n_batches);

/* Run the Z-shape stage over the current plan (pipeline_ggr.hpp:119-134): per
 * batch refresh_cost, Z-shape DP and traceback (zshape::solve, reset_nodes,
 * convert_routes) into the route words, ++stamp, thread-per-net wire then via
 * commit (commit_wire_demand / commit_via_demand, demand.cuh:129-232).  The
 * reference's host post-processing (promote_congested_segments,
 * canonicalize_routes) stays with the caller. */
int grb_zshape_stage(grb_ctx* ctx, int32_t mode, grb_stats* stats);

/* ---- Differentiable routing cost (no counterpart in the reference) ------- */
#define GRB_F32 0
#define GRB_F64 1

/* Soft-min L-shape DAG: the DP of Lshape_route (lshape_thread.cuh:18-171)
 * over every uploaded net with each min replaced by
 * smin(v) = -tau * log(sum exp(-v / tau)), on cost tables computed in the
 * working precision from `capacity` and the per-edge `unit_wire` cost
 * (device arrays of L*X*Y floats or doubles, per dtype) at the context's
 * current demand (full_update.cuh:9-83 without float narrowing).  Writes each
 * net's soft cost to net_cost (device, n values) and their sum to *total.
 * As tau -> 0 the value tends to the hard DP's optimum. */
int grb_softmin_forward(grb_ctx* ctx, int32_t dtype, double tau, const void* capacity, const void* unit_wire,
                        double unit_via, void* net_cost, double* total);
/* Hand-written adjoint of grb_softmin_forward: grad_total * d(total)/d(capacity)
 * into dcap, d(total)/d(unit_wire) per edge into dunit_wire (device arrays
 * like the inputs) and d(total)/d(unit_via) into *dunit_via.  Each net's DP
 * tables are recomputed in a per-thread slot (memory bounded by the threads
 * in flight, not by the nets); as tau -> 0 the gradient tends to the
 * indicator of the chosen routes. */
int grb_softmin_backward(grb_ctx* ctx, int32_t dtype, double tau, const void* capacity, const void* unit_wire,
                         double unit_via, double grad_total, void* dcap, void* dunit_wire, double* dunit_via);

/* Stage tail: the rip-up classification (flags bit 0, GRB_TAIL_RIPUP, with
 * graph::ripup's threshold) and the congestion view (bit 1, GRB_TAIL_VIEW) of
 * the final demand, computed by every following grb_lshape_stage right after
 * its last batch -- in the persistent executor inside the same kernel, with
 * no host round trip between the stage and them (the reference runs both
 * right after its L-shape stage, pipeline.hpp:86-93, each with a host
 * synchronisation; the rip-up flags it then downloads, flt.cuh:58-60, are
 * read here with grb_read_stage_tail).  flags = 0 turns the tail off.
 * Allocates its buffers here (one int per cell, one byte per net, a byte and
 * two floats per 2-D cell). */
#define GRB_TAIL_RIPUP 1
#define GRB_TAIL_VIEW 2
int grb_set_stage_tail(grb_ctx* ctx, int32_t flags, int32_t threshold);
/* Copy the last stage tail's results to the host: is_of[n] (as
 * grb_ripup_classify), congestion/xsum/ysum[X*Y] (as grb_congestion_view);
 * any pointer may be NULL. */
int grb_read_stage_tail(grb_ctx* ctx, uint8_t* is_of, uint8_t* congestion, float* xsum, float* ysum);

/* Congestion view for the FLT topology builder (congestion.cuh:60-112). */
int grb_congestion_view(grb_ctx* ctx, uint8_t* congestion, float* xsum, float* ysum);

/* The cost model's exponential as the cost kernels evaluate it on `device`
 * (CUDA's __expf on a float argument, the reference's choice in
 * full_update.cuh:12-13): y[i] = exp(x[i]) for n host values (no counterpart
 * in the reference).  For checkers that restate the cost model on the host and
 * must reproduce the device's cost tables bit for bit: given these values for
 * the arguments the model can produce, a host restatement needs no copy of the
 * device's exponential.  Needs no context; allocates and synchronises. */
int grb_cost_exp(int32_t device, const float* x, int32_t n, float* y);

/* Read device tables (any pointer may be NULL). */
int grb_read_tables(grb_ctx* ctx, float* wcost, float* vcost, double* presum, int32_t* demand_half,
                    int32_t* timestamp);
/* Copy all route words (route_off[n] words) to the host. */
int grb_read_routes(grb_ctx* ctx, int32_t* routes);
/* Copy only the route words in use: for each net, its count word r[0] and
 * the words below it (at least the count word), to the same offsets of
 * `routes`; every other word of `routes` is left as it was.  A route holds a
 * small part of its reserved storage (the GGR build reserves 256 words per pin,
 * pipeline_ggr.hpp:9), so this moves a small part of what download_routes
 * copies (router_state.hpp:215-222); host code that reads a route only below
 * its count -- the GGR post-processing, zshape_topology.hpp:122-248, and the
 * writer -- sees the same routes. */
int grb_read_routes_used(grb_ctx* ctx, int32_t* routes);
/* The reverse of grb_read_routes_used: for each net, the count word at its
 * offset of `routes` (clamped to the net's storage) and the words below it are
 * written to the device; the device's other words keep their values. */
int grb_write_routes_used(grb_ctx* ctx, const int32_t* routes);
/* Replace all route words (route_off[n] words) from the host: routes a caller
 * edited after a stage (the GGR pipeline's promote_congested_segments and
 * canonicalize_routes, zshape_topology.hpp:122-248) for grb_format_out.
 * Demand and timestamps are left as they are. */
int grb_write_routes(grb_ctx* ctx, const int32_t* routes);
int grb_get_stats(grb_ctx* ctx, grb_stats* stats);
/* Set the statistics counters (the reference uploads RouterState::statistics,
 * whose via count starts at the number of metal1 pins, preprocess.hpp:1716-1718
 * and :1780). */
int grb_set_stats(grb_ctx* ctx, double total_wirelength, int64_t total_via_count);
/* Wait for the context's stream and report any recorded device error. */
int grb_sync(grb_ctx* ctx);

/* Number of kernels this context has launched so far (graph launches count
 * every kernel node); used for launch accounting by callers. */
int64_t grb_kernel_launches(grb_ctx* ctx);

/* Limit of every device-side wait of the persistent kernels (grid barriers
 * and the batching kernel's hand-over counters), in seconds; 20 by default.
 * A wait that runs out records GRB_ETIMEDOUT, every block of the kernel
 * returns, and the call that launched it reports GRB_ETIMEDOUT.  The
 * context's tables are then in an unspecified state: grb_reset (and a new
 * plan) before the next stage.  (The reference has no device waits.) */
int grb_set_wait_limit(grb_ctx* ctx, double seconds);

/* Profiling (off by default).  When on, the plain form brackets each launch
 * group with CUDA events and the persistent kernels time each phase between
 * grid barriers (global timer, thread 0 of one block).  grb_phase_times
 * returns accumulated milliseconds per phase (up to 20 entries):
 * batching [0] raster (persistent: publish of the previous chunk), [1]
 * gather of forbidden colours and predecessors (persistent: gather of the
 * next chunk and raster of the one after), [2] in-chunk solve, [3] publish
 * (plain form only); stages [4] cost recompute of the dirty chunks with
 * prefix pass 1, [5] DP (persistent: + wire commit), [6] commit
 * (persistent: vias), [7] prefix trees and pass 2; persistent batching [8]
 * solver waiting for a gathered chunk, [9] other blocks waiting for a solved
 * chunk; [10] and [11] unused; persistent L-shape stage, per size bucket k of
 * the DP (tree nodes <= 2, <= 8, <= 16, more): [12+k] warp time summed over
 * its nets, [16+k] the longest single net (a maximum, not a sum).  The reference prints its stage timings as BATCH_TIMING /
 * DAG_TIMING records (router_state.hpp:259-264). */
int grb_set_profiling(grb_ctx* ctx, int32_t on);
int grb_phase_times(grb_ctx* ctx, double* ms, int32_t n, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif
