/*
 * grb_prof.h -- measurement helpers of grotor_b200 (host side, no GPU work).
 */
#ifndef GRB_PROF_H
#define GRB_PROF_H
#include <stdint.h>
#include "grb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Algorithmic (compulsory) bytes of one L-shape stage over a plan, by part:
 * out[0] cost refresh: 12 B per dirty wire cell (capacity + demand read, wcost
 *        write), 20 B per dirty via cell, 12 B per element of every dirty track
 *        (4 B read + 8 B prefix write); the first batch counts every cell/track;
 * out[1] DP: 8 B per distinct prefix entry and 4 B per distinct via-cost entry a
 *        net reads, 8 B per tree node (node + parent word), 4 B per route word;
 * out[2] commit: 12 B per wire unit edge (demand read-modify-write + timestamp),
 *        8 B per via half-update;
 * out[3] batching: 4 B per query point, 4 B per marked cell, 132 B per net
 *        (colour mask + batch id).
 * routes are the stage's route words; ids/batch_off its plan. */
int grb_stage_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                      const int32_t* node_off, const int32_t* nodes, const int32_t* parents,
                      const int64_t* route_off, const int32_t* routes,
                      const int32_t* point_off, const int32_t* hseg_off, const int32_t* hsegs,
                      const int32_t* vseg_off, const int32_t* vsegs, int32_t sparsity, double* out);

/* The same model for the Z-shape stage (grb_zshape_stage) over its plan and
 * trees: out[0] refresh, out[2] commit as above; out[1] DP: per net 8 B per
 * distinct prefix entry and 4 B per distinct via-cost entry it reads (for a
 * tree edge with a bend, the two rows and two columns of its box on every
 * layer; for a straight edge its end points on the layers of its direction;
 * every node's via column), 16 B per node, 4 B per route word. */
int grb_zshape_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                       const int32_t* node_off, const int32_t* coord, const int32_t* child,
                       const int64_t* route_off, const int32_t* routes, double* out);

/* The same model for the FLT stage (grb_flt_stage): per batch, with
 * remove_phase_one, the commit bytes of removing the nets' stage-one routes
 * (routes at route_off), then refresh, DP and the commit of the phase-two
 * routes (routes2 at dags->route2_off).  DP: per net 8 B per distinct prefix
 * entry and 4 B per distinct via-cost entry it reads (each edge's straight
 * wires and its sampled layer changes), 20 B per node, 8 B per edge, 4 B per
 * route word. */
int grb_flt_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                    const grb_flt_dags* dags, const int64_t* route_off, const int32_t* routes, const int32_t* routes2,
                    int32_t remove_phase_one, double* out);

/* The L-shape DP's read set, summed over nets ids[0..n) (all nets when ids is
 * NULL): out[0] distinct prefix entries, out[1] distinct via-cost entries,
 * out[2] tree nodes.  The soft-min DAG reads the same entries. */
int grb_dag_reads(const grb_grid* g, int32_t n, const int32_t* ids, const int32_t* node_off, const int32_t* nodes,
                  const int32_t* parents, double* out);

#ifdef __cplusplus
}
#endif
#endif
