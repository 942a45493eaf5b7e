/*
 * grb_synth.h -- seeded synthetic CAP/NET designs and their routing topology.
 *
 * Host-side workload preparation for grotor_b200 (not part of the routing hot
 * path).  The generator draws ISPD-2024-style designs (a GCell grid with edge
 * capacities and nets of pins); the topology builder turns every net into the
 * inputs the reference's stage drivers hand to the GPU: nets above 12 pins
 * split into subnets (preprocess.hpp:1448-1623 splits at MAX_PIN_SIZE = 12),
 * a rectilinear Steiner tree per subnet in DFS order from node 0
 * (lshape.cuh:85-103), and the batching geometry of net::construct_rsmt
 * (preprocess.hpp:88-130).  The reference builds its trees with FLUTE, which
 * is not part of this repository; this builder is a rectilinear MST with
 * greedy median Steiner points.  Designs can be written as CAP/NET files that
 * the reference router reads unchanged.
 */
#ifndef GRB_SYNTH_H
#define GRB_SYNTH_H
#include <stdint.h>
#include "grb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct grb_design grb_design;

typedef struct grb_synth_params {
    int32_t X, Y;
    int32_t cap_layers;        /* CAP layers; routing layers L = cap_layers - 1 */
    int32_t n_nets;
    int32_t cap_lo, cap_hi;    /* capacity uniform integer in [cap_lo, cap_hi] */
    double blockage;           /* fraction of (x,y) cells with capacity 0 on every layer */
    double unit_wire, unit_via, overflow_weight;
    int32_t pin_model;         /* 0: two_pin_frac two-pin, else 3 + Geometric(geo_p) <= max_pins;
                                  1: 2 + floor(Lomax(pareto_alpha)) <= max_pins */
    double two_pin_frac, geo_p;
    int32_t max_pins;
    double pareto_alpha;
    int32_t bbox_model;        /* 0: round(LogNormal(ln median, sigma)), big_frac nets with side U[big_lo, big_hi];
                                  1: round(exp(U(0, ln bbox_max))) */
    double bbox_median, bbox_sigma, big_frac;
    int32_t big_lo, big_hi, bbox_max;
    int32_t pin_cap_layers;    /* pins on CAP layers U{0 .. pin_cap_layers-1} */
    uint64_t seed;
} grb_synth_params;

grb_design* grb_synth_generate(const grb_synth_params* p);
void grb_design_free(grb_design* d);
const char* grb_design_error(const grb_design* d);

/* Grid of the design (pointers owned by the design). */
int grb_design_grid(const grb_design* d, grb_grid* out);
/* Write the design as reference CAP and NET files. */
int grb_design_write(const grb_design* d, const char* cap_path, const char* net_path);

/* Build subnets and trees (threads <= 0: all host threads). */
int grb_design_build_topology(grb_design* d, int32_t max_subnet_pins, int32_t threads);
/* Topology arrays (owned by the design, valid until the next build or free). */
int grb_design_nets(const grb_design* d, grb_nets* out);
/* The same trees in the Z-shape encoding (grb_zshape_trees): preorder from
 * each tree's first leaf, children in ascending node order; a node with more
 * than three children hands the extra ones to the nearest node with room in
 * its first child's subtree (built on the first call; owned by the design). */
int grb_design_zshape_trees(grb_design* d, const int32_t** node_off, const int32_t** coord, const int32_t** child);
/* Per-subnet HPWL, original net id and pin count (arrays of n entries). */
int grb_design_subnet_info(const grb_design* d, const int32_t** hpwl, const int32_t** original,
                           const int32_t** pin_count);
/* Nets ordered by HPWL, largest first, ties by id (the stage order, lshape.cuh:53-55). */
int grb_design_order(const grb_design* d, int32_t* order);
/* Raw nets: pins as CAP-layer cell ids l*X*Y + x*Y + y, CSR by net. */
int grb_design_pins(const grb_design* d, const int32_t** pin_off, const int32_t** pins, int32_t* n_nets);

#ifdef __cplusplus
}
#endif
#endif
