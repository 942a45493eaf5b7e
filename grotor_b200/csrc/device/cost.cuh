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

// The exponential of the cost model: CUDA's __expf on a float argument, the
// reference's choice (full_update.cuh:12-13).  grb_cost_exp evaluates the same
// function for checkers.
__device__ __forceinline__ float cost_exp(float a) { return __expf(a); }

__device__ __forceinline__ double of_cost_scaled(double scale, float capacity, float demand) {
    if (capacity > 0.001) {
        const float diff = demand - capacity;
        return cost_exp(static_cast<float>(fmin(0.5 * diff, scale * 0.5 * diff)));
    }
    if (demand > 0) return cost_exp(static_cast<float>(fmin(1.5 * demand, scale * 1.5 * demand)));
    return 0;
}

// Cost terms of one cell: the overflow increments of adding a whole unit
// and half a unit of demand (incremental_of_cost with incre 1.0 and 0.5, in
// its arithmetic; the exponential of the current demand is shared).
__device__ __forceinline__ void cell_terms(const Tables& T, float cap, int dem_half, double sc, double& one,
                                           double& half) {
    const float dem = static_cast<float>(dem_half) * 0.5f;
    const float w1 = static_cast<float>(static_cast<double>(dem) + 1.0 + 0.0);
    const float wh = static_cast<float>(static_cast<double>(dem) + 0.5 + 0.0);
    const float w0 = static_cast<float>(static_cast<double>(dem) + 0.0);
    const double o0 = of_cost_scaled(T.of_scale, cap, w0);
    one = fmin(1e12, (of_cost_scaled(T.of_scale, cap, w1) - o0) * sc);
    half = fmin(1e12, (of_cost_scaled(T.of_scale, cap, wh) - o0) * sc);
}

// The terms the cost kernels use per cell: `wof`, the overflow increment of
// a whole unit rounded to float (what the wire cost and the end-of-track via
// cost start from) and `half`, the increment of half a unit (double, what an
// interior via cost sums).
__device__ __forceinline__ double2 terms_of(double one, double half) {
    return make_double2(static_cast<double>(static_cast<float>(one)), half);
}

// Computed from capacity and demand (out of line: the table below covers
// almost every cell, and the refresh's unrolled loops stay small).
__device__ __noinline__ double2 cell_terms_computed(const Tables& T, int c, int dem_half, double sc) {
    double one, half;
    cell_terms(T, T.capacity[c], dem_half, sc, one, half);
    return terms_of(one, half);
}

// The terms of cell c (capacity row cid, demand dem_half half-units) on a
// layer of weight sc.  The demands the cost model evaluates are h/2, h/2 + 1/2
// and h/2 + 1 (exactly (h+1)/2 and (h+2)/2 in float), so for a capacity with a
// table row and a demand in range the terms are precomputed per (layer,
// capacity, demand) by the same functions: the same bits.
__device__ __forceinline__ double2 cell_terms_at(const Tables& T, int l, int c, unsigned cid, int dem_half,
                                                 double sc) {
    if (cid != kNoCapRow && dem_half >= 0 && dem_half < T.of_dmax)
        return __ldg(T.of_table + (size_t(l) * T.of_rows + cid) * T.of_stride + dem_half);
    return cell_terms_computed(T, c, dem_half, sc);
}

// update_single_wcost_ispd24 (full_update.cuh:34-51) from the cell's terms;
// the length term is the fused multiply-add the compiler forms for
// `w += unit * len`.  elen: the edge length (ignored at the track's end).
__device__ __forceinline__ float wire_cost_of(const Tables& T, double wof, int pos, int len, int elen) {
    float w = static_cast<float>(wof);
    if (pos < len - 1) w = static_cast<float>(fma(T.unit_wire, static_cast<double>(elen), wof));
    // The GGR build keeps integer DP edges non-negative and below its sentinel
    // (full_update.cuh:47-50).
    if (T.int_wire) w = static_cast<float>(static_cast<long long>(fminf(fmaxf(w, 0.f), 1.e7f)));
    return w;
}

// update_single_vcost_ispd24 (full_update.cuh:58-83) from the terms of the
// cell and of the previous cell along its track; cross points are zero on a
// single GPU (preprocess.hpp:1757).
__device__ __forceinline__ float via_cost_of(const Tables& T, const double2& t, const double2& prev, int pos,
                                             int len) {
    float v;
    if (pos == 0) v = static_cast<float>(t.x);
    else if (pos == len - 1) v = static_cast<float>(prev.x);
    else v = static_cast<float>(t.y + prev.y);
    return static_cast<float>(static_cast<double>(v) + T.unit_via);
}

// What the costs of cell c depend on: its own terms and those of the
// previous cell along its track (capacity row and demand of each), its
// position, the track length and the edge length.
struct CellInputs {
    unsigned cid0, cid1;
    int dem0, dem1;
    int l, pos, len, elen, stride;
};

__device__ __forceinline__ CellInputs load_cell(const Tables& T, int c) {
    CellInputs in;
    const int l = c / T.XY, rem = c - l * T.XY, x = rem / T.Y, y = rem - x * T.Y;
    const bool ay = along_y(T, l);
    in.l = l;
    in.stride = ay ? 1 : T.Y;
    in.pos = ay ? y : x;
    in.len = ay ? T.Y : T.X;
    in.cid0 = T.cap_id[c];
    in.dem0 = T.demand[c];
    in.cid1 = in.pos > 0 ? T.cap_id[c - in.stride] : 0u;
    in.dem1 = in.pos > 0 ? T.demand[c - in.stride] : 0;
    in.elen = in.pos < in.len - 1 ? (ay ? T.ylen[in.pos] : T.xlen[in.pos]) : 0;
    return in;
}

// Position of the n-th (0-based) set bit of m, which has more than n set
// bits: a binary search over halves, quarters, ... by population count, the
// same few instructions for every lane whatever n is.
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w; w >>= 1) {
        const unsigned low = m & ((1u << w) - 1u);
        const int c = __popc(low);
        const bool up = n >= c;
        n = up ? n - c : n;
        pos = up ? pos + w : pos;
        m = up ? m >> w : low;
    }
    return pos;
}

// update_dirty_costs / update_dirty_wire_cost (incremental_update.cuh:44-96):
// recompute every dirty cell.  A warp loads 32 bitmap words at a time, ranks
// their dirty cells with a warp prefix sum and takes them kRounds * 32 at a
// time, kRounds cells per lane whose inputs are all loaded before any cost is
// computed or stored (kRounds trades registers for loads in flight).  Wire
// costs where the wire bit is set, via costs where the via bit is set (a
// wire-dirty cell is always via-dirty); the terms come from the cost-term
// table.  Both words are cleared.  `warp`/`nwarps` number the calling warps
// across the launch.
template <int kRounds>
__device__ __forceinline__ void refresh_dirty_cells(const Tables& T, int warp, int nwarps, int lane) {
    // The next window's bitmap words are loaded while this one is processed.
    int nw = warp * 32 + lane;
    unsigned nvb = nw < T.words ? T.dirty_via[nw] : 0u;
    unsigned nwb = nw < T.words ? T.dirty_wire[nw] : 0u;
    for (int base = warp * 32; base < T.words; base += nwarps * 32) {
        const int w = base + lane;
        const unsigned vb = nvb, wb = nwb;
        nw = w + nwarps * 32;
        nvb = nw < T.words ? T.dirty_via[nw] : 0u;
        nwb = nw < T.words ? T.dirty_wire[nw] : 0u;
        const int n = __popc(vb);
        int incl = n;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int r = 0; r < total; r += 32 * kRounds) {
            int cell[kRounds];
            bool wire[kRounds];
#pragma unroll
            for (int q = 0; q < kRounds; ++q) {
                const int k = r + q * 32 + lane;
                // Owner lane: first lane whose inclusive count exceeds k.
                int lo = 0;
#pragma unroll
                for (int step = 16; step; step >>= 1) {
                    const int v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
                    if (v <= k) lo += step;
                }
                const int owner_incl = __shfl_sync(0xffffffffu, incl, lo);
                const int owner_n = __shfl_sync(0xffffffffu, n, lo);
                const unsigned ov = __shfl_sync(0xffffffffu, vb, lo), ow = __shfl_sync(0xffffffffu, wb, lo);
                cell[q] = -1;
                wire[q] = false;
                if (k < total) {
                    const int nth = k - (owner_incl - owner_n);  // 0-based rank inside the owner's word
                    const int bit = nth_set_bit(ov, nth);
                    const int c = (base + lo) * 32 + bit;
                    if (c < T.cells) {
                        cell[q] = c;
                        wire[q] = (ow >> bit) & 1u;
                    }
                }
            }
            CellInputs in[kRounds];
#pragma unroll
            for (int q = 0; q < kRounds; ++q)
                if (cell[q] >= 0) in[q] = load_cell(T, cell[q]);
#pragma unroll
            for (int q = 0; q < kRounds; ++q) {
                if (cell[q] < 0) continue;
                const int c = cell[q];
                const double sc = T.short_costs[in[q].l];
                const double2 t0 = cell_terms_at(T, in[q].l, c, in[q].cid0, in[q].dem0, sc);
                const double2 t1 = in[q].pos > 0
                                       ? cell_terms_at(T, in[q].l, c - in[q].stride, in[q].cid1, in[q].dem1, sc)
                                       : make_double2(0.0, 0.0);
                if (wire[q]) T.wcost[c] = wire_cost_of(T, t0.x, in[q].pos, in[q].len, in[q].elen);
                T.vcost[c] = via_cost_of(T, t0, t1, in[q].pos, in[q].len);
            }
        }
        if (vb) T.dirty_via[w] = 0u;
        if (wb) T.dirty_wire[w] = 0u;
    }
}

// Prefix rebuild.  A group is 32 adjacent tracks of one layer (one per lane);
// positions are cut into aligned 32-position chunks.  Work items are (group,
// chunk) pairs, one warp each, spread over the whole GPU:
//   pass 1: each lane runs the reference association over its chunk (stack of
//           aligned block totals, fully unrolled into registers) and stores the
//           chunk total (level 0 of the group's tree, global memory);
//   tree:   one CTA per group builds the totals of aligned 2^e-chunk blocks,
//           pairwise (level e entry b = level e-1 entries 2b+1 + 2b);
//   pass 2: each lane re-runs its chunk, and every element adds, lowest bit
//           first, the totals of the aligned blocks below it at levels >= 5.
// The result equals the reference's per-track scan bit for bit.  Wire costs
// must be current (refresh_dirty_cells runs first).
constexpr int kChunkPos = 32;

__host__ __device__ __forceinline__ int prefix_chunks(int len) { return (len + kChunkPos - 1) / kChunkPos; }
__host__ __device__ __forceinline__ int prefix_tree_entries(int len) { return 2 * prefix_chunks(len) + 1; }
__host__ __device__ __forceinline__ size_t prefix_smem_bytes(int max_len) {
    return size_t(prefix_tree_entries(max_len)) * 32 * sizeof(double);
}

// Per-warp shared scratch of the passes: a 32 x 32 chunk of doubles (rows
// padded to 33 entries so row and column accesses are conflict-free).
constexpr int kXposeStride = kChunkPos + 1;
__host__ __device__ __forceinline__ size_t prefix_xpose_bytes() {
    return size_t(kTrackGroup) * kXposeStride * sizeof(double);
}

struct GroupGeom {
    int l, len, nch, base, stride;
    bool live;
};

__device__ __forceinline__ GroupGeom group_geom(const Tables& T, int g, int lane) {
    GroupGeom G;
    int l = 0;
    while (l + 1 <= T.L && g >= T.group_base[l + 1]) ++l;
    const bool ay = along_y(T, l);
    const int tracks = ay ? T.X : T.Y;
    const int track = (g - T.group_base[l]) * kTrackGroup + lane;
    G.l = l;
    G.len = ay ? T.Y : T.X;
    G.nch = prefix_chunks(G.len);
    G.live = track < tracks;
    G.base = ay ? cell_index(T, l, G.live ? track : 0, 0) : cell_index(T, l, 0, G.live ? track : 0);
    G.stride = ay ? 1 : T.Y;
    return G;
}

// The shifted input s[i] = w[i-1] of chunk c (0 outside the track); wire
// costs are floats, widened when used.  Along-x tracks: at each position the
// 32 lanes read 32 consecutive cells.  Along-y tracks are runs of consecutive
// cells, one per lane; with scratch `xs` the warp reads them run by run (32
// consecutive floats per instruction) and transposes through shared memory.
__device__ __forceinline__ void load_chunk(const Tables& T, const GroupGeom& G, int c, float (&x)[kChunkPos],
                                           int lane, float* xs) {
    const int i0 = c * kChunkPos;
    if (xs && G.stride == 1) {
        const int i = i0 + lane;
        // Rows in groups of 16, every load of a group issued before its
        // shared-memory stores.
#pragma unroll
        for (int r0 = 0; r0 < kTrackGroup; r0 += 16) {
            float v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int base = __shfl_sync(0xffffffffu, G.base, r0 + r);
                const int live = __shfl_sync(0xffffffffu, int(G.live), r0 + r);
                v[r] = (live && i > 0 && i < G.len) ? T.wcost[base + i - 1] : 0.0f;
            }
#pragma unroll
            for (int r = 0; r < 16; ++r) xs[(r0 + r) * kXposeStride + lane] = v[r];
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < kChunkPos; ++k) x[k] = xs[lane * kXposeStride + k];
        __syncwarp();
        return;
    }
#pragma unroll
    for (int k = 0; k < kChunkPos; ++k) {
        const int i = i0 + k;
        x[k] = (G.live && i > 0 && i < G.len) ? T.wcost[G.base + (i - 1) * G.stride] : 0.0f;
    }
}

// The pairwise total of a chunk's prefix inputs: the reference association
// over the chunk (k = 31 has all five low bits set, so the final accumulator
// is the total of the aligned 32-block).
__device__ __forceinline__ double chunk_total(const float (&x)[kChunkPos]) {
    double tot[6];
    double acc = 0;
#pragma unroll
    for (int k = 0; k < kChunkPos; ++k) {
        acc = static_cast<double>(x[k]);
        double fresh[6];
        fresh[0] = acc;
        int t = 0;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            if (((k >> d) & 1) && ((k & ((1 << d) - 1)) == (1 << d) - 1)) {
                acc = acc + tot[d];
                fresh[d + 1] = acc;
                t = d + 1;
            }
        }
#pragma unroll
        for (int d = 0; d < 6; ++d) if (d <= t) tot[d] = fresh[d];
    }
    return acc;
}

// Pass 1 for work item (g, c): the chunk total of every lane's track (wire
// costs must be current).  `xs`: the warp's scratch (prefix_xpose_bytes), or
// null.
__device__ __forceinline__ void prefix_pass1(const Tables& T, int g, int c, int lane, void* xs) {
    const GroupGeom G = group_geom(T, g, lane);
    float x[kChunkPos];
    load_chunk(T, G, c, x, lane, static_cast<float*>(xs));
    T.ptree[(size_t(g) * T.tree_stride + c) * 32 + lane] = chunk_total(x);
}

// Tree of aligned block totals for group g (one CTA, `tree` = shared memory
// of prefix_smem_bytes): level 0 from global, higher levels built here, the
// whole tree written back.
__device__ __forceinline__ void prefix_tree(const Tables& T, int g, double* tree) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const GroupGeom G = group_geom(T, g, lane);
    double* gt = T.ptree + size_t(g) * T.tree_stride * 32;
    for (int c = warp; c < G.nch; c += nwarp) tree[c * 32 + lane] = gt[c * 32 + lane];
    __syncthreads();
    int off = 0, cnt = G.nch;
    while (cnt > 1) {
        const int up = cnt >> 1;
        for (int b = warp; b < up; b += nwarp) {
            const double v = tree[(off + 2 * b + 1) * 32 + lane] + tree[(off + 2 * b) * 32 + lane];
            tree[(off + cnt + b) * 32 + lane] = v;
            gt[(off + cnt + b) * 32 + lane] = v;
        }
        __syncthreads();
        off += cnt;
        cnt = up;
    }
}

// Final prefix values of chunk c from its prefix inputs x and the totals
// add[e] of the aligned blocks of 2^e chunks below it (for the set bits e of
// c; 0 elsewhere): per element, lowest bit first, the blocks inside the chunk
// then the chunk-level blocks.  Along-y tracks with scratch `xs`: the values
// go through shared memory and are written run by run (32 consecutive
// doubles per instruction).
__device__ __forceinline__ void chunk_prefix_store(const Tables& T, const GroupGeom& G, int c,
                                                   const float (&x)[kChunkPos], const double (&add)[8], int lane,
                                                   void* xs) {
    const bool rows = xs && G.stride == 1;
    double* ds = static_cast<double*>(xs);
    double tot[6];
    const int i0 = c * kChunkPos;
#pragma unroll
    for (int k = 0; k < kChunkPos; ++k) {
        double acc = static_cast<double>(x[k]);
        double fresh[6];
        fresh[0] = acc;
        int t = 0;
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            if (((k >> d) & 1) && ((k & ((1 << d) - 1)) == (1 << d) - 1)) {
                acc = acc + tot[d];
                fresh[d + 1] = acc;
                t = d + 1;
            }
        }
#pragma unroll
        for (int d = 0; d < 6; ++d) if (d <= t) tot[d] = fresh[d];
#pragma unroll
        for (int e = 0; e < 5; ++e)
            if (e > t && ((k >> e) & 1)) acc = acc + tot[e];
#pragma unroll
        for (int e = 0; e < 8; ++e)
            if ((c >> e) & 1) acc = acc + add[e];
        const int i = i0 + k;
        if (rows) ds[lane * kXposeStride + k] = acc;
        else if (G.live && i < G.len) T.presum[G.base + i * G.stride] = acc;
    }
    if (rows) {
        __syncwarp();
        const int i = i0 + lane;
#pragma unroll
        for (int r0 = 0; r0 < kTrackGroup; r0 += 16) {
            double v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = ds[(r0 + r) * kXposeStride + lane];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int base = __shfl_sync(0xffffffffu, G.base, r0 + r);
                const int live = __shfl_sync(0xffffffffu, int(G.live), r0 + r);
                if (live && i < G.len) T.presum[base + i] = v[r];
            }
        }
        __syncwarp();
    }
}

// Pass 2 for work item (g, c): final prefix values of the chunk, its inputs
// re-read from the wire costs and the chunk-level totals from the tree.
__device__ __forceinline__ void prefix_pass2(const Tables& T, int g, int c, int lane, void* xs) {
    const GroupGeom G = group_geom(T, g, lane);
    const double* gt = T.ptree + size_t(g) * T.tree_stride * 32;
    double add[8];
    {
        int off = 0, cnt = G.nch;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            add[e] = 0.0;
            if (cnt >= 1 && ((c >> e) & 1)) add[e] = gt[(off + (c >> e) - 1) * 32 + lane];
            off += cnt;
            cnt >>= 1;
        }
    }
    float x[kChunkPos];
    load_chunk(T, G, c, x, lane, static_cast<float*>(xs));
    chunk_prefix_store(T, G, c, x, add, lane, xs);
}

// Move the dirty groups (group_first below INT_MAX) into group_list and mark
// them clean (one CTA).  The commits that follow mark them again for the next
// refresh.
__device__ __forceinline__ void collect_dirty_groups(const Tables& T) {
    __shared__ int count;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    for (int g = threadIdx.x; g < T.n_groups; g += blockDim.x) {
        const int first = T.group_first[g];
        if (first != 0x7fffffff) {
            const int k = atomicAdd(&count, 1);
            T.group_list[k] = g;
            T.first_list[k] = first;
            T.group_first[g] = 0x7fffffff;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *T.group_count = count;
}

// Work items (k, c): chunk c of the k-th dirty group, enumerated as
// k * tree_chunks + c.  Chunks before the group's first changed chunk keep
// their prefix values and their level-0 totals from the previous rebuild.
__device__ __forceinline__ bool prefix_item(const Tables& T, int item, int& g, int& c) {
    const int k = item / T.tree_chunks;
    c = item - k * T.tree_chunks;
    if (k >= *reinterpret_cast<const volatile int*>(T.group_count)) return false;
    if (c < T.first_list[k]) return false;
    g = T.group_list[k];
    int l = 0;
    while (l + 1 <= T.L && g >= T.group_base[l + 1]) ++l;
    return c < prefix_chunks(along_y(T, l) ? T.Y : T.X);
}

}  // namespace grb
