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

#ifdef __cplusplus
}
#endif
#endif
