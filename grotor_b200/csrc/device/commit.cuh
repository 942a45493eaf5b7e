// commit.cuh -- demand commit and rip-up of routed nets.
//
// Semantics of the reference's batch commit (demand.cuh:236-319): wires first
// (each unit edge gets K, its timestamp becomes the batch stamp, both segment
// endpoints are stamped), then -- after every wire of the batch is in -- vias:
// each via layer whose cell was not stamped by a wire of this batch adds K to
// its single neighbouring edge at a track end, else K/2 to the two edges it
// lands between.  K = -1 removes a route.  Half-unit integer demand makes every
// update exact and order-free, so warps may commit in any order.
#pragma once
#include "common.cuh"

namespace grb {

__device__ __forceinline__ const int* net_routes(const Plan& P, int id) { return P.routes + P.route_off[id]; }

// One warp commits the wire segments of net `id` (of `parts` warps sharing a
// net, warp `part` takes every parts-th segment); lanes split each segment's
// unit edges.  Along-y segments cover consecutive cells, so their dirty bits
// are set a bitmap word at a time (fenwick.cuh:51-78).
__device__ __forceinline__ void commit_net_wires(const Tables& T, const Plan& P, int id, int stamp, int K,
                                                 int lane, int part = 0, int parts = 1) {
    const int* r = net_routes(P, id);
    const int words = r[0];
    double length = 0;
    for (int i = 1 + 2 * part; i < words; i += 2 * parts) {
        const int a = r[i], b = r[i + 1], layer = a / T.XY;
        if (layer != b / T.XY) continue;
        const int ra = a - layer * T.XY, rb = b - layer * T.XY;
        const int x0 = ra / T.Y, y0 = ra - x0 * T.Y, x1 = rb / T.Y, y1 = rb - x1 * T.Y;
        const bool ay = x0 == x1;
        const int lo = ay ? min(y0, y1) : min(x0, x1), hi = ay ? max(y0, y1) : max(x0, x1);
        if (lane == 0) {
            T.ts[a] = stamp;
            T.ts[b] = stamp;
            if (hi > lo) {
                mark_group_dirty(T, layer, ay ? x0 : y0, lo);
                if (ay) {
                    const int first = layer * T.XY + x0 * T.Y + lo;
                    mark_range(T.dirty_wire, first, first + (hi - lo) - 1);
                    mark_range(T.dirty_via, first, first + (hi - lo));
                }
            }
        }
        for (int pos = lo + lane; pos < hi; pos += 32) {
            const int c = layer * T.XY + (ay ? x0 * T.Y + pos : pos * T.Y + y0);
            red_add(T.demand + c, 2 * K);
            T.ts[c] = stamp;
            if (!ay) {
                set_bits(T.dirty_wire, c >> 5, 1u << (c & 31));
                set_bits(T.dirty_via, c >> 5, 1u << (c & 31));
                if (pos + 1 < T.X) set_bits(T.dirty_via, (c + T.Y) >> 5, 1u << ((c + T.Y) & 31));
            }
            length += ay ? T.ylen[pos] : T.xlen[pos];
        }
    }
    for (int s = 16; s; s >>= 1) length += __shfl_down_sync(0xffffffffu, length, s);
    if (lane == 0 && length != 0.0) atomicAdd(T.wirelength, length * K);
}

// Via demand on cell c, position pos of track `track` of layer l.
__device__ __forceinline__ void add_via_demand(const Tables& T, int c, int half, int l, int track, int pos, int len,
                                               int stride) {
    red_add(T.demand + c, half);
    mark_edge_dirty(T, c, l, track, pos, len, stride);
}

// Demand of the via stack at (x, y) (ra = x*Y + y) between layers low and
// high: every layer whose cell no wire of this batch stamped adds K at a track
// end, else K/2 to the two edges it lands between.  All timestamps of the
// stack are loaded before the first update.
__device__ __forceinline__ void via_stack_demand(const Tables& T, int ra, int x, int y, int low, int high, int stamp,
                                                 int K) {
    int ts[kMaxLayers];
#pragma unroll
    for (int u = 0; u < kMaxLayers; ++u) ts[u] = low + u < high ? T.ts[(low + u) * T.XY + ra] : stamp;
#pragma unroll
    for (int u = 0; u < kMaxLayers; ++u) {
        const int layer = low + u;
        if (layer >= high || ts[u] >= stamp) continue;
        const int c = layer * T.XY + ra;
        const bool ay = along_y(T, layer);
        const int pos = ay ? y : x, len = ay ? T.Y : T.X, stride = ay ? 1 : T.Y, track = ay ? x : y;
        if (!pos) add_via_demand(T, c, 2 * K, layer, track, pos, len, stride);
        else if (pos == len - 1) add_via_demand(T, c - stride, 2 * K, layer, track, pos - 1, len, stride);
        else {
            add_via_demand(T, c - stride, K, layer, track, pos - 1, len, stride);
            add_via_demand(T, c, K, layer, track, pos, len, stride);
        }
    }
}

// Route segment (a, b): if it is a via, commit its stack and return the
// number of layers it crosses, else 0.
__device__ __forceinline__ int via_segment(const Tables& T, int a, int b, int stamp, int K) {
    const int la = a / T.XY, lb = b / T.XY;
    const int low = min(la, lb), high = max(la, lb);
    if (low == high) return 0;
    const int ra = a - la * T.XY, x = ra / T.Y, y = ra - x * T.Y;
    via_stack_demand(T, ra, x, y, low, high, stamp, K);
    return high - low;
}

// One warp commits the via segments of the nets ids[first], ids[first +
// step], ... below ids[cnt] (routes of plan P), lanes over each net's
// segments.  The warp loads the ids and route offsets of 32 of
// its nets at once, and each net's first 32 segments (those inside its route
// capacity) while the previous net's via stacks are committed, so a net costs
// about one memory round trip instead of four.
__device__ __forceinline__ void commit_vias_strided(const Tables& T, const Plan& P, const int* ids, int cnt,
                                                    int first, int step, int stamp, int K, int lane) {
    long long vias = 0;
    for (int g0 = first; g0 < cnt; g0 += 32 * step) {
        const int mine = g0 + lane * step;
        long long off = 0, cap = 0;
        if (mine < cnt) {
            const int id = ids[mine];
            off = P.route_off[id];
            cap = P.route_off[id + 1] - off;
        }
        const int nn = min(32, (cnt - 1 - g0) / step + 1);
        const int i0 = 1 + 2 * lane;
        // Net j's word count and lane's first segment (if inside capacity).
        int words = 0, a = 0, b = 0;
        {
            const int* r = P.routes + __shfl_sync(0xffffffffu, off, 0);
            const long long c = __shfl_sync(0xffffffffu, cap, 0);
            words = r[0];
            if (i0 + 1 < c) { a = r[i0]; b = r[i0 + 1]; }
        }
        for (int j = 0; j < nn; ++j) {
            const int* r = P.routes + __shfl_sync(0xffffffffu, off, j);
            const long long c = __shfl_sync(0xffffffffu, cap, j);
            const int cw = words, ca = a, cb = b;
            if (j + 1 < nn) {
                const int* rn = P.routes + __shfl_sync(0xffffffffu, off, j + 1);
                const long long nc = __shfl_sync(0xffffffffu, cap, j + 1);
                words = rn[0];
                if (i0 + 1 < nc) { a = rn[i0]; b = rn[i0 + 1]; }
            }
            if (i0 < cw) vias += i0 + 1 < c ? via_segment(T, ca, cb, stamp, K) : via_segment(T, r[i0], r[i0 + 1], stamp, K);
            for (int i = i0 + 64; i < cw; i += 64) vias += via_segment(T, r[i], r[i + 1], stamp, K);
        }
    }
    for (int s = 16; s; s >>= 1) vias += __shfl_down_sync(0xffffffffu, vias, s);
    if (lane == 0 && vias) atomicAdd(T.vias, static_cast<unsigned long long>(vias * K));
}

// Thread-per-net forms (commit_wire_demand / commit_via_demand,
// demand.cuh:129-232), used where the reference commits one net per thread
// (the Z-shape stage).  Same demand, timestamps, dirty marks and statistics as
// the warp forms above.
__device__ __forceinline__ void commit_thread_wires(const Tables& T, const Plan& P, int id, int stamp, int K) {
    const int* r = net_routes(P, id);
    const int words = r[0];
    double length = 0;
    for (int i = 1; i < words; i += 2) {
        const int a = r[i], b = r[i + 1], layer = a / T.XY;
        if (layer != b / T.XY) continue;
        const int ra = a - layer * T.XY, rb = b - layer * T.XY;
        const int x0 = ra / T.Y, y0 = ra - x0 * T.Y, x1 = rb / T.Y, y1 = rb - x1 * T.Y;
        const bool ay = x0 == x1;
        const int lo = ay ? min(y0, y1) : min(x0, x1), hi = ay ? max(y0, y1) : max(x0, x1);
        T.ts[a] = stamp;
        T.ts[b] = stamp;
        if (hi > lo) {
            mark_group_dirty(T, layer, ay ? x0 : y0, lo);
            if (ay) {
                const int first = layer * T.XY + x0 * T.Y + lo;
                mark_range(T.dirty_wire, first, first + (hi - lo) - 1);
                mark_range(T.dirty_via, first, first + (hi - lo));
            }
        }
        for (int pos = lo; pos < hi; ++pos) {
            const int c = layer * T.XY + (ay ? x0 * T.Y + pos : pos * T.Y + y0);
            red_add(T.demand + c, 2 * K);
            T.ts[c] = stamp;
            if (!ay) {
                set_bits(T.dirty_wire, c >> 5, 1u << (c & 31));
                set_bits(T.dirty_via, c >> 5, 1u << (c & 31));
                if (pos + 1 < T.X) set_bits(T.dirty_via, (c + T.Y) >> 5, 1u << ((c + T.Y) & 31));
            }
            length += ay ? T.ylen[pos] : T.xlen[pos];
        }
    }
    if (length != 0.0) atomicAdd(T.wirelength, length * K);
}

__device__ __forceinline__ void commit_thread_vias(const Tables& T, const Plan& P, int id, int stamp, int K) {
    const int* r = net_routes(P, id);
    const int words = r[0];
    long long vias = 0;
    for (int i = 1; i < words; i += 2) {
        const int a = r[i], b = r[i + 1];
        const int la = a / T.XY, lb = b / T.XY;
        const int low = min(la, lb), high = max(la, lb);
        if (low == high) continue;
        const int ra = a - la * T.XY, x = ra / T.Y, y = ra - x * T.Y;
        vias += high - low;
        via_stack_demand(T, ra, x, y, low, high, stamp, K);
    }
    if (vias) atomicAdd(T.vias, static_cast<unsigned long long>(vias * K));
}

}  // namespace grb
