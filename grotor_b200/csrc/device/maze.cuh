// maze.cuh -- the device steps of the CUGR2 pipeline's maze stage.
//
// Semantics (pipeline_cugr2.hpp:90-117, maze.cuh:9-64, maze_quality.cuh:8-43):
//   * remove_routes: every listed net's current route leaves the demand and
//     the statistics -- each wire unit edge -1, and each via layer whose cell
//     none of the net's own wires covers (net-local membership, so bulk
//     removal of overlapping nets needs no timestamps) -1 at a track end,
//     else -1/2 on the two edges it lands between; the statistics lose the
//     net's edge lengths and via layers;
//   * routing_score: wirelength * unit wire cost + vias * unit via cost + the
//     overflow cost of every edge cell, summed by a fixed tree (1024 blocks of
//     256 threads, each thread over cells t, t + 262144, ..., then a block
//     halving tree, then the 1024 partials in order on the host), so the
//     acceptance test of a rerouted stage does not depend on atomic order.
#pragma once
#include "commit.cuh"
#include "cost.cuh"

namespace grb {

// A wire of route r (words [1, r[0])) on point's layer covers point.
__device__ __forceinline__ bool maze_wire_touches(const int* r, int point, int XY, int Y) {
    const int layer = point / XY;
    for (int i = 1; i < r[0]; i += 2) {
        const int a = r[i], b = r[i + 1];
        if (a / XY != layer || b / XY != layer) continue;
        const int x = point / Y, y = point % Y;  // x carries the layer offset, as a / Y does
        if (a % Y == y && b % Y == y && x >= min(a / Y, b / Y) && x <= max(a / Y, b / Y)) return true;
        if (a / Y == x && b / Y == x && y >= min(a % Y, b % Y) && y <= max(a % Y, b % Y)) return true;
    }
    return false;
}

// Edge cell c of layer l changes by `half` half-units (and is marked dirty).
__device__ __forceinline__ void maze_add(const Tables& T, int c, int half) {
    const int l = c / T.XY, r = c - l * T.XY, x = r / T.Y, y = r - x * T.Y;
    const bool ay = along_y(T, l);
    add_via_demand(T, c, half, l, ay ? x : y, ay ? y : x, ay ? T.Y : T.X, ay ? 1 : T.Y);
}

// remove_routes for one net (one thread): route words r.
__device__ __forceinline__ void maze_remove_route(const Tables& T, const int* r) {
    const int XY = T.XY, Y = T.Y, X = T.X;
    double length = 0;
    long long vias = 0;
    for (int i = 1; i < r[0]; i += 2) {
        const int a = r[i], b = r[i + 1];
        const int x = a / Y % X, y = a % Y;
        if (a / XY == b / XY) {
            const int base = a / XY * XY, bx = b / Y % X, by = b % Y;
            for (int xx = min(x, bx); xx < max(x, bx); ++xx) {
                maze_add(T, base + xx * Y + y, -2);
                length += T.xlen[xx];
            }
            for (int yy = min(y, by); yy < max(y, by); ++yy) {
                maze_add(T, base + x * Y + yy, -2);
                length += T.ylen[yy];
            }
        } else {
            const int first = min(a / XY, b / XY), last = max(a / XY, b / XY);
            vias += last - first;
            for (int layer = first; layer < last; ++layer) {
                const int point = layer * XY + x * Y + y;
                if (maze_wire_touches(r, point, XY, Y)) continue;
                const bool vertical = along_y(T, layer);
                const int position = vertical ? y : x, limit = vertical ? Y : X, step = vertical ? 1 : Y;
                if (!position) maze_add(T, point, -2);
                else if (position == limit - 1) maze_add(T, point - step, -2);
                else {
                    maze_add(T, point - step, -1);
                    maze_add(T, point, -1);
                }
            }
        }
    }
    if (length != 0.0) atomicAdd(T.wirelength, -length);
    if (vias) atomicAdd(T.vias, static_cast<unsigned long long>(-vias));
}

constexpr int kScoreBlocks = 1024, kScoreThreads = 256;

// One block's partial of the overflow cost (maze_quality.cuh:8-26 order).
__device__ __forceinline__ void maze_score_partial(const Tables& T, double* partials) {
    __shared__ double sums[kScoreThreads];
    const size_t cells = size_t(T.L) * T.XY;
    double value = 0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < cells; i += size_t(gridDim.x) * blockDim.x) {
        const int layer = int(i / T.XY), x = int(i / T.Y % T.X), y = int(i % T.Y);
        if (along_y(T, layer) ? y + 1 < T.Y : x + 1 < T.X)
            value += T.short_costs[layer] * of_cost_scaled(1.0, T.capacity[i], 0.5f * static_cast<float>(T.demand[i]));
    }
    sums[threadIdx.x] = value;
    __syncthreads();
    for (int stride = kScoreThreads / 2; stride; stride /= 2) {
        if (threadIdx.x < stride) sums[threadIdx.x] += sums[threadIdx.x + stride];
        __syncthreads();
    }
    if (!threadIdx.x) partials[blockIdx.x] = sums[0];
}

}  // namespace grb
