// common.cuh -- device-side state view and shared helpers for the routing path.
//
// Grid layout follows the reference router (router_state.hpp:267):
// IDX(l,x,y) = (l*X + x)*Y + y, and layer l carries wires along y when
// ((l & 1) ^ DIR) is 1, along x otherwise.  Demand is int32 half-units: a wire
// edge adds 2, a split via landing adds 1 to each neighbour (demand.cuh:300-304
// uses 1.0f and 0.5f), so demand * 0.5f reproduces the reference's float.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace grb {

constexpr double kInf = 1e22;   // router_state.hpp:271
constexpr int kMaxLayers = 10;  // lshape_warp.cuh:115 asserts L <= 10
constexpr int kTrackGroup = 32; // tracks per prefix group (one per lane)
constexpr int kNoCapRow = 255;  // cap_id of a cell whose capacity has no table row

enum : int {
    kOk = 0, kEInval = 1, kENoMem = 2, kECuda = 3, kETimedOut = 4, kELimit = 5,
};

// Device tables of one routing context.  Copied by value into every kernel.
struct Tables {
    int L, X, Y, DIR, XY;
    int cells;
    double unit_wire, unit_via, of_scale;
    const double* short_costs;
    const int* xlen;
    const int* ylen;
    const float* capacity;
    int* demand;           // half-units
    int* ts;               // commit timestamps
    float* wcost;
    float* vcost;
    double* presum;
    unsigned* dirty_wire;  // one bit per cell: wire cost to recompute
    unsigned* dirty_via;   // one bit per cell: via cost to recompute
    int words;             // bitmap words
    int int_wire;          // 1: wire costs clamped to [0, 1e7] and truncated (GGR build)
    // Cost-term table: row (l, k) holds, for demands h < of_dmax half-units,
    // the terms of a cell of capacity value k on layer l (cost.cuh
    // cell_terms_at); one row per layer and distinct capacity value (cap_id[c]
    // = k of cell c, kNoCapRow where the design has too many values).
    const unsigned char* cap_id;
    const double2* of_table;
    int of_rows;           // capacity values (rows per layer)
    int of_stride;         // entries per row
    int of_dmax;           // demands below this come from the table
    // Prefix groups: kTrackGroup adjacent tracks of one layer.  A group's
    // prefix is rebuilt from the first 32-position chunk where a wire cost of
    // one of its tracks changed.
    int group_base[kMaxLayers + 1];
    int* group_first;      // [n_groups] first chunk with a demand change (INT_MAX: none)
    int* first_list;       // [n_groups] group_first of each listed dirty group
    int n_groups;
    int* group_list;       // [n_groups] dirty groups of the current refresh
    int* group_count;      // [1]
    double* ptree;         // [n_groups][tree_stride][32] prefix block totals
    int tree_stride;       // entries per group (2 * tree_chunks + 1)
    int tree_chunks;       // 32-position chunks of the longest track
    double* wirelength;
    unsigned long long* vias;
    int* error;            // first error code
    int* error_info;       // detail (net index, ...)
};

// Topology of the current plan (device pointers).
struct Plan {
    const int* node_off;       // [n_nets+1], indexed by net id
    const int* nodes;          // l*X*Y + x*Y + y, l == L for Steiner nodes
    const int* parents;        // parent < child, -1 at the root
    const long long* route_off;// [n_nets+1] word offsets into routes
    int* routes;               // [count, a0, b0, ...] per net
    const int* ids;            // net ids in execution order
    const int* batch_off;      // [n_batches+1] into ids
    int n_batches;
    // The same plan with each batch's nets grouped by size bucket
    // (kDpBuckets): bucket_ids, and per batch kDpBuckets+1 offsets into it.
    const int* bucket_ids;
    const int* bucket_off;
};

// Size buckets of the routing DP: tree nodes <= 2 (routed one net per lane),
// <= 8, <= 16, more (one net per warp).
constexpr int kDpBuckets = 4;
__host__ __device__ __forceinline__ int dp_bucket(int nodes) {
    return nodes <= 2 ? 0 : nodes <= 8 ? 1 : nodes <= 16 ? 2 : 3;
}
__host__ __device__ __forceinline__ int dp_bucket_nodes(int b) { return b == 0 ? 2 : b == 1 ? 8 : 16; }

// Launch shape chosen per size bucket (grb_autotune): nets per CTA of the
// per-batch DP launch, nets taken per work-queue grab in the persistent form.
struct DpTune {
    int per_cta[kDpBuckets];
    int per_grab[kDpBuckets];
};

__device__ __forceinline__ bool along_y(const Tables& T, int l) { return ((l & 1) ^ T.DIR) != 0; }
__device__ __forceinline__ int cell_index(const Tables& T, int l, int x, int y) { return (l * T.X + x) * T.Y + y; }

__device__ __forceinline__ void set_error(const Tables& T, int code, int info) {
    if (atomicCAS(T.error, 0, code) == 0) *T.error_info = info;
}

// Fire-and-forget reductions: the result is never read, so the instruction
// carries no return value and the issuing thread does not wait for L2.
__device__ __forceinline__ void red_or(unsigned* p, unsigned v) {
    asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_add(int* p, int v) {
    asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_min(int* p, int v) {
    asm volatile("red.relaxed.gpu.global.min.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void set_bits(unsigned* bits, int word, unsigned mask) {
    if (mask) red_or(bits + word, mask);
}

// A wire cost of track `track` of layer l at position `pos` changed: the
// group's prefix must be rebuilt from that position's 32-position chunk on.
__device__ __forceinline__ void mark_group_dirty(const Tables& T, int l, int track, int pos) {
    red_min(T.group_first + T.group_base[l] + track / kTrackGroup, pos >> 5);
}

// A demand change on edge cell c (position pos of track `track` of layer l,
// track length len, stride along the track) invalidates its wire cost, its
// own via cost and the via cost of the next cell along the track
// (fenwick.cuh:27-38).
__device__ __forceinline__ void mark_edge_dirty(const Tables& T, int c, int l, int track, int pos, int len,
                                                int stride) {
    set_bits(T.dirty_wire, c >> 5, 1u << (c & 31));
    set_bits(T.dirty_via, c >> 5, 1u << (c & 31));
    if (pos + 1 < len) set_bits(T.dirty_via, (c + stride) >> 5, 1u << ((c + stride) & 31));
    mark_group_dirty(T, l, track, pos);
}

// Mark cells [first, last] of a bitmap with one atomic per word
// (fenwick.cuh:40-49).
__device__ __forceinline__ void mark_range(unsigned* bits, int first, int last) {
    const int a = first >> 5, b = last >> 5;
    for (int w = a; w <= b; ++w) {
        unsigned m = ~0u;
        if (w == a) m &= ~0u << (first & 31);
        if (w == b) m &= ~0u >> (31 - (last & 31));
        set_bits(bits, w, m);
    }
}

// Grid-wide barrier for cooperative launches: one monotone arrival counter
// (zeroed before the launch).  Barrier k of a launch completes when the
// counter reaches k * gridDim.x, so no reset or generation word is needed and
// a barrier costs one acquire-release atomic plus acquire polls.  Every wait
// is bounded by the global timer; on expiry the kernel records kETimedOut and
// callers return.  `epoch` counts this block's barriers (a kernel-local copy).
struct GridSync {
    unsigned* count;
    unsigned* generation;          // unused by the counter barrier
    unsigned long long timeout_ns;
    unsigned long long* phase_ns;  // optional per-phase time accumulators
    unsigned epoch;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0 waits until *p >= target: relaxed polls (an acquire load per poll
// would invalidate the SM's L1 under the warps still working), backing off
// after the first polls so long waits do not flood the word's L2 slice, then
// one fence so later reads see the writes that preceded the producers'
// releases.  Gives up, recording kETimedOut, after timeout_ns; also returns
// false as soon as any error is recorded when `any_error` is set (the
// producer may have stopped), else only on a timeout elsewhere.
__device__ __forceinline__ bool wait_at_least(const unsigned* p, unsigned target, unsigned long long timeout_ns,
                                              const Tables& T, bool any_error) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    if (v < target) {
        const unsigned long long start = global_ns();
        unsigned spins = 0;
        while (v < target) {
            if ((++spins & 63) == 0) {
                if (global_ns() - start > timeout_ns) { set_error(T, kETimedOut, blockIdx.x); return false; }
                const int e = *reinterpret_cast<volatile int*>(T.error);
                if (any_error ? e != 0 : e == kETimedOut) return false;
            }
            if (spins > 16) __nanosleep(spins > 256 ? 128 : 32);
            asm volatile("ld.relaxed.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        }
    }
    __threadfence();  // acquire: later reads see every producer's writes
    return true;
}

// Barrier of `members` blocks (every block of the grid, or a subset that
// shares the counter); barrier k completes at k * members arrivals.
__device__ __forceinline__ bool grid_sync_of(GridSync& s, const Tables& T, unsigned members) {
    __shared__ int ok;
    const unsigned target = (++s.epoch) * members;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned v;
        __threadfence();
        asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(v) : "l"(s.count) : "memory");
        ok = v + 1 >= target ? 1 : wait_at_least(s.count, target, s.timeout_ns, T, false);
        if (v + 1 >= target) __threadfence();
    }
    __syncthreads();
    return ok != 0;
}
__device__ __forceinline__ bool grid_sync(GridSync& s, const Tables& T) { return grid_sync_of(s, T, gridDim.x); }

struct PhaseClock {
    unsigned long long last = 0;
    int owner = 0;  // the block whose thread 0 records
    __device__ __forceinline__ void start(const GridSync& s) {
        if (s.phase_ns && blockIdx.x == owner && threadIdx.x == 0) last = global_ns();
    }
    __device__ __forceinline__ void mark(const GridSync& s, int k) {
        if (s.phase_ns && blockIdx.x == owner && threadIdx.x == 0) {
            const unsigned long long now = global_ns();
            s.phase_ns[k] += now - last;
            last = now;
        }
    }
};

}  // namespace grb
