// cost.cuh -- per-edge congestion cost and per-track prefix tables.
//
// Cost formulas follow the reference's cost model (full_update.cuh:9-83) in
// the same arithmetic: float demand/capacity differences, double scaling,
// CUDA's __expf on a float argument, a double difference weighted per layer,
// stored as float.  The prefix table is the reference's double per-track
// prefix (prefix_scan.cuh:74-114, fenwick.cuh:129-168): presum[i] sums the
// shifted track [0, w0, w1, ...] in the same association (for each set bit d of
// i, lowest first, add the pairwise total of the aligned 2^d block below), so
// every presum value is bit-identical to the reference's.
//
// B200 layout: a prefix "group" is 32 adjacent tracks of one layer.  One CTA of
// 256 threads owns a group and walks it in chunks of 64 positions; a thread
// holds 8 consecutive positions of one track, so a warp touches 32 adjacent
// tracks at the same positions (along-x layers: 32 consecutive y, one 128-byte
// line per position) or 8-element runs of 32 rows (along-y layers).  The
// reference launches one CTA per single track with stride-Y accesses.
#pragma once
#include "common.cuh"

namespace grb {

__device__ __forceinline__ double of_cost_scaled(double scale, float capacity, float demand) {
    if (capacity > 0.001) {
        const float diff = demand - capacity;
        return __expf(fmin(0.5 * diff, scale * 0.5 * diff));
    }
    if (demand > 0) return __expf(fmin(1.5 * demand, scale * 1.5 * demand));
    return 0;
}

__device__ __forceinline__ double incremental_of_cost(const Tables& T, int c, int l, double incre) {
    const float cap = T.capacity[c];
    const float dem = static_cast<float>(T.demand[c]) * 0.5f;
    const float with = static_cast<float>(static_cast<double>(dem) + incre + 0.0);
    const float without = static_cast<float>(static_cast<double>(dem) + 0.0);
    return fmin(1e12, (of_cost_scaled(T.of_scale, cap, with) - of_cost_scaled(T.of_scale, cap, without)) *
                          T.short_costs[l]);
}

// update_single_wcost_ispd24 (full_update.cuh:34-51); the length term is the
// fused multiply-add the compiler forms for `w += unit * len`.
__device__ __forceinline__ float wire_cost_at(const Tables& T, int c) {
    const int l = c / T.XY, rem = c - l * T.XY, x = rem / T.Y, y = rem - x * T.Y;
    float w = static_cast<float>(incremental_of_cost(T, c, l, 1.0));
    if (!along_y(T, l) && x < T.X - 1) w = static_cast<float>(fma(T.unit_wire, static_cast<double>(T.xlen[x]), static_cast<double>(w)));
    if (along_y(T, l) && y < T.Y - 1) w = static_cast<float>(fma(T.unit_wire, static_cast<double>(T.ylen[y]), static_cast<double>(w)));
    return w;
}

// update_single_vcost_ispd24 (full_update.cuh:58-83); cross points are zero
// on a single GPU (preprocess.hpp:1757).
__device__ __forceinline__ float via_cost_at(const Tables& T, int c) {
    const int l = c / T.XY, rem = c - l * T.XY, x = rem / T.Y, y = rem - x * T.Y;
    float v;
    if (along_y(T, l)) {
        if (y == 0) v = static_cast<float>(incremental_of_cost(T, c, l, 1.0));
        else if (y == T.Y - 1) v = static_cast<float>(incremental_of_cost(T, c - 1, l, 1.0));
        else v = static_cast<float>(incremental_of_cost(T, c, l, 0.5) + incremental_of_cost(T, c - 1, l, 0.5));
    } else {
        if (x == 0) v = static_cast<float>(incremental_of_cost(T, c, l, 1.0));
        else if (x == T.X - 1) v = static_cast<float>(incremental_of_cost(T, c - T.Y, l, 1.0));
        else v = static_cast<float>(incremental_of_cost(T, c, l, 0.5) + incremental_of_cost(T, c - T.Y, l, 0.5));
    }
    return static_cast<float>(static_cast<double>(v) + T.unit_via);
}

// Recompute the via costs of one dirty bitmap word (32 consecutive cells);
// one warp, one lane per cell.  The word is cleared afterwards.
__device__ __forceinline__ void refresh_via_word(const Tables& T, int w, int lane) {
    const unsigned bits = T.dirty_via[w];
    const int c = w * 32 + lane;
    if (((bits >> lane) & 1u) && c < T.cells) T.vcost[c] = via_cost_at(T, c);
    __syncwarp();
    if (lane == 0) T.dirty_via[w] = 0;
}

// Rebuild the prefix of one group (CTA-wide, blockDim.x == 256).  When
// `recompute` is set, dirty wire cells read on the way are recomputed first
// (the persistent executor fuses the cost update into the scan).
template <bool recompute>
__device__ void refresh_group(const Tables& T, int g, double* stack /* smem [32][16] */,
                              double* t3 /* smem [8][32] */) {
    int l = 0;
    while (l + 1 <= T.L && g >= T.group_base[l + 1]) ++l;
    const bool ay = along_y(T, l);
    const int tracks = ay ? T.X : T.Y, len = ay ? T.Y : T.X;
    const int track0 = (g - T.group_base[l]) * kTrackGroup;
    const int lane = threadIdx.x & 31, sub = threadIdx.x >> 5;
    const int track = track0 + lane;
    const bool live = track < tracks;
    const int base = ay ? cell_index(T, l, track < tracks ? track : 0, 0) : cell_index(T, l, 0, track < tracks ? track : 0);
    const int stride = ay ? 1 : T.Y;
    double* my_stack = stack + lane * 16;
    for (int p0 = 0; p0 < len; p0 += 64) {
        const int i0 = p0 + sub * 8;
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = i0 + k;
            double x = 0.0;
            if (live && i > 0 && i < len) {
                const int c = base + (i - 1) * stride;
                float w;
                if (recompute && bit_test(T.dirty_wire, c)) {
                    w = wire_cost_at(T, c);
                    T.wcost[c] = w;
                    atomicAnd(T.dirty_wire + (c >> 5), ~(1u << (c & 31)));
                } else {
                    w = T.wcost[c];
                }
                x = static_cast<double>(w);
            }
            v[k] = x;
        }
        if (recompute && live && i0 <= len - 1 && len - 1 < i0 + 8) {
            // The last cell of a track feeds no prefix entry but keeps its cost current.
            const int c = base + (len - 1) * stride;
            if (bit_test(T.dirty_wire, c)) {
                T.wcost[c] = wire_cost_at(T, c);
                atomicAnd(T.dirty_wire + (c >> 5), ~(1u << (c & 31)));
            }
        }
        // Levels 0..2 inside the aligned 8-run (sum[i] += sum[(i>>d<<d)-1]).
        v[1] = v[1] + v[0]; v[3] = v[3] + v[2]; v[5] = v[5] + v[4]; v[7] = v[7] + v[6];
        v[2] = v[2] + v[1]; v[3] = v[3] + v[1]; v[6] = v[6] + v[5]; v[7] = v[7] + v[5];
        v[4] = v[4] + v[3]; v[5] = v[5] + v[3]; v[6] = v[6] + v[3]; v[7] = v[7] + v[3];
        t3[sub * 32 + lane] = v[7];
        __syncthreads();
        // Levels 3..5: totals of aligned 8-, 16- and 32-runs below this run.
        double add3 = 0, add4 = 0, add5 = 0;
        if (sub & 1) add3 = t3[(sub - 1) * 32 + lane];
        if (sub & 2) {
            const int q = (sub >> 1) - 1;  // 16-run index below
            add4 = t3[(2 * q + 1) * 32 + lane] + t3[(2 * q) * 32 + lane];
        }
        if (sub & 4) {
            const double up = t3[3 * 32 + lane] + t3[2 * 32 + lane];
            const double lo = t3[1 * 32 + lane] + t3[0 * 32 + lane];
            add5 = up + lo;
        }
        // Levels >= 6: completed 64-aligned blocks below this chunk.
        const int chunk = p0 >> 6;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            double acc = v[k];
            if (sub & 1) acc = acc + add3;
            if (sub & 2) acc = acc + add4;
            if (sub & 4) acc = acc + add5;
            for (int e = 0; (chunk >> e) != 0; ++e)
                if ((chunk >> e) & 1) acc = acc + my_stack[e];
            const int i = i0 + k;
            if (live && i < len) T.presum[base + i * stride] = acc;
            v[k] = acc;
        }
        __syncthreads();
        // Push this chunk's total (element 63 before the high levels) onto the
        // per-track stack of completed block totals.
        if (sub == 7) {
            double up = t3[7 * 32 + lane] + t3[6 * 32 + lane];
            up = up + (t3[5 * 32 + lane] + t3[4 * 32 + lane]);
            const double lo = (t3[3 * 32 + lane] + t3[2 * 32 + lane]) + (t3[1 * 32 + lane] + t3[0 * 32 + lane]);
            double total = up + lo;
            double fresh[16];
            fresh[0] = total;
            int d = 0;
            while ((chunk >> d) & 1) {
                total = total + my_stack[d];
                ++d;
                fresh[d] = total;
            }
            for (int j = 0; j <= d; ++j) my_stack[j] = fresh[j];
        }
        __syncthreads();
    }
}

}  // namespace grb
