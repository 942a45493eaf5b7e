// congestion.cuh -- rip-up classification and congestion view of the
// committed demand (the reference's graph::ripup and extract_congestionView*,
// congestion.cuh:8-136).  Device functions shared by the standalone kernels
// and by the tail of the persistent L-shape stage.
#pragma once
#include "common.cuh"

namespace grb {

// mark_overflow_edges (congestion.cuh:8-20): 1 where the edge of cell c
// carries demand >= capacity + threshold (cells without an edge: 0).
__device__ __forceinline__ void overflow_mark(const Tables& T, int threshold, int* of_sum, int c) {
    const int l = c / T.XY, rem = c - l * T.XY, x = rem / T.Y, y = rem - x * T.Y;
    const bool edge = along_y(T, l) ? (y + 1 < T.Y) : (x + 1 < T.X);
    of_sum[c] = (edge && T.capacity[c] + threshold <= static_cast<float>(T.demand[c]) * 0.5f) ? 1 : 0;
}

// Exclusive integer prefix of the marks along track t (all layers' tracks
// numbered consecutively; compute_presum_general, prefix_scan.cuh:42-72 --
// integer sums are order-free).
__device__ __forceinline__ void overflow_prefix_track(const Tables& T, int* v, int t) {
    int l = 0, base = t;
    for (; l < T.L; ++l) {
        const int tracks = along_y(T, l) ? T.X : T.Y;
        if (base < tracks) break;
        base -= tracks;
    }
    if (l >= T.L) return;
    const bool ay = along_y(T, l);
    const int len = ay ? T.Y : T.X, stride = ay ? 1 : T.Y;
    const int c0 = ay ? cell_index(T, l, base, 0) : cell_index(T, l, 0, base);
    int acc = 0;
    for (int k = 0; k < len; ++k) {
        const int c = c0 + k * stride, x = v[c];
        v[c] = acc;
        acc += x;
    }
}

__device__ __forceinline__ int overflow_tracks(const Tables& T) {
    int tracks = 0;
    for (int l = 0; l < T.L; ++l) tracks += along_y(T, l) ? T.X : T.Y;
    return tracks;
}

// mark_overflow_nets (congestion.cuh:22-58): net `id` is flagged when its
// wires cross more than 10 overflowing edges.
__device__ __forceinline__ unsigned char overflow_route(const Tables& T, const int* r, bool has, const int* of_sum) {
    int count = 0;
    unsigned char flag = 0;
    if (has) {
        for (int i = 1; i < r[0]; i += 2) {
            const int a = r[i], b = r[i + 1], l = a / T.XY, ra = a % T.XY, rb = b % T.XY;
            const int x0 = ra / T.Y, y0 = ra % T.Y, x1 = rb / T.Y, y1 = rb % T.Y;
            if (x0 != x1) count += of_sum[cell_index(T, l, max(x0, x1), y0)] - of_sum[cell_index(T, l, min(x0, x1), y0)];
            if (y0 != y1) count += of_sum[cell_index(T, l, x0, max(y0, y1))] - of_sum[cell_index(T, l, x0, min(y0, y1))];
            if (count > 10) { flag = 1; break; }
        }
    }
    return flag;
}
__device__ __forceinline__ void overflow_net(const Tables& T, const Plan& P, const int* of_sum, unsigned char* is_of,
                                             int id) {
    is_of[id] = overflow_route(T, P.routes + P.route_off[id], P.route_off[id + 1] > P.route_off[id], of_sum);
}

// extract_congestionView (congestion.cuh:60-80) for 2-D cell i: the worst
// demand - capacity over the layers.
__device__ __forceinline__ void congestion_cell(const Tables& T, unsigned char* cong, float* xsum, float* ysum,
                                                int i) {
    double worst = 0.0;
    for (int l = 0; l < T.L; ++l) {
        const int e = l * T.XY + i;
        worst = fmax(worst, static_cast<double>(static_cast<float>(T.demand[e]) * 0.5f - T.capacity[e]));
    }
    cong[i] = worst > 0.0;
    xsum[i] = static_cast<float>(worst);
    ysum[i] = static_cast<float>(worst);
}

// Float prefix of one line (extract_congestionView_xsum / _ysum,
// congestion.cuh:81-112): the shifted line [0, v0, v1, ...] summed in the
// reference's log-step association (for each set bit of i, lowest first, the
// total of the aligned block below), one thread per line.
__device__ __forceinline__ void congestion_line_prefix(float* a, int len, int elem_stride) {
    float tot[32];
    float prev = 0.f;
    for (int i = 0; i < len; ++i) {
        const float cur = a[size_t(i) * elem_stride];
        float acc = i ? prev : 0.f;
        prev = cur;
        float fresh[32];
        fresh[0] = acc;
        int d = 0;
        while ((i >> d) & 1) { acc = acc + tot[d]; ++d; fresh[d] = acc; }
        for (int j = 0; j <= d; ++j) tot[j] = fresh[j];
        for (int e = d + 1; (i >> e) != 0; ++e)
            if ((i >> e) & 1) acc = acc + tot[e];
        a[size_t(i) * elem_stride] = acc;
    }
}

// What the tail of an L-shape stage computes from the final demand
// (pipeline.hpp:86-93 runs the congestion view and graph::ripup right after
// the stage): flags bit 0 = rip-up classification, bit 1 = congestion view.
enum : int { kTailRipup = 1, kTailView = 2 };
struct StageTail {
    int flags;
    int threshold;
    int n_nets;
    int* of_sum;            // [cells]
    unsigned char* is_of;   // [n_nets]
    unsigned char* cong;    // [X*Y]
    float* xsum;            // [X*Y]
    float* ysum;            // [X*Y]
};

// The stage tail inside a persistent kernel (grid-stride over all threads):
// marks and per-cell view | track prefixes and line prefixes | net flags,
// separated by grid barriers.  False when a barrier gave up.
__device__ __forceinline__ bool stage_tail_persistent(const Tables& T, const Plan& P, const StageTail& tail,
                                                      GridSync& S) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (tail.flags & kTailRipup)
        for (int c = tid; c < T.cells; c += nth) overflow_mark(T, tail.threshold, tail.of_sum, c);
    if (tail.flags & kTailView)
        for (int i = tid; i < T.XY; i += nth) congestion_cell(T, tail.cong, tail.xsum, tail.ysum, i);
    if (!grid_sync(S, T)) return false;
    if (tail.flags & kTailRipup) {
        const int tracks = overflow_tracks(T);
        for (int t = tid; t < tracks; t += nth) overflow_prefix_track(T, tail.of_sum, t);
    }
    if (tail.flags & kTailView) {
        // per x along y (ysum), then per y along x (xsum), one thread per line
        for (int t = tid; t < T.X + T.Y; t += nth) {
            if (t < T.X) congestion_line_prefix(tail.ysum + size_t(t) * T.Y, T.Y, 1);
            else congestion_line_prefix(tail.xsum + (t - T.X), T.X, T.Y);
        }
    }
    if (!grid_sync(S, T)) return false;
    if (tail.flags & kTailRipup)
        for (int id = tid; id < tail.n_nets; id += nth) overflow_net(T, P, tail.of_sum, tail.is_of, id);
    return true;
}

}  // namespace grb
