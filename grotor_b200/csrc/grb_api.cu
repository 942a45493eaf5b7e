// grb_api.cu -- C ABI, routing context and executors (plain, CUDA graph,
// persistent) of the B200 routing hot path.
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/grb.h"
#include "device/batching.cuh"
#include "device/commit.cuh"
#include "device/congestion.cuh"
#include "device/common.cuh"
#include "device/cost.cuh"
#include "device/flt.cuh"
#include "device/outfmt.cuh"
#include "device/lshape.cuh"
#include "device/maze.cuh"
#include "device/softmin.cuh"
#include "device/topology.cuh"
#include "device/zshape.cuh"

using namespace grb;

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
namespace {

constexpr int kRefreshThreads = 256;       // threads of a prefix-tree CTA
constexpr int kPersistentThreads = 256;
constexpr int kDpThreads = 128;
constexpr unsigned long long kBarrierTimeoutNs = 20ull * 1000 * 1000 * 1000;
constexpr int kPhaseSlots = 20;  // grb_phase_times entries
constexpr int kNetTimeSlot = 12;  // per size bucket: summed net time [12..15], longest net [16..19]

// update_dirty_costs (incremental_update.cuh:62-96): recompute dirty cells.
__global__ void k_refresh_cells(Tables T) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    refresh_dirty_cells<4>(T, warp, nwarps, lane);
}

// Prefix rebuild of dirty groups: pass 1 and pass 2 over (group, chunk) work
// items, one warp each; the tree with one CTA per group.
__global__ void k_collect_groups(Tables T) { collect_dirty_groups(T); }
__global__ void __launch_bounds__(256, 2) k_prefix_pass1(Tables T) {
    extern __shared__ __align__(16) char xsm[];
    void* xs = xsm + (threadIdx.x >> 5) * prefix_xpose_bytes();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int items = *T.group_count * T.tree_chunks;
    for (int item = warp; item < items; item += nwarps) {
        int g, c;
        if (prefix_item(T, item, g, c)) prefix_pass1(T, g, c, lane, xs);
    }
}
__global__ void __launch_bounds__(kRefreshThreads) k_prefix_tree(Tables T) {
    extern __shared__ __align__(16) double tree[];
    for (int k = blockIdx.x; k < *T.group_count; k += gridDim.x) prefix_tree(T, T.group_list[k], tree);
}
__global__ void __launch_bounds__(256, 2) k_prefix_pass2(Tables T) {
    extern __shared__ __align__(16) char xsm[];
    void* xs = xsm + (threadIdx.x >> 5) * prefix_xpose_bytes();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int items = *T.group_count * T.tree_chunks;
    for (int item = warp; item < items; item += nwarps) {
        int g, c;
        if (prefix_item(T, item, g, c)) prefix_pass2(T, g, c, lane, xs);
    }
}

// Everything dirty: the state of a fresh database (first refresh is full).
__global__ void k_mark_all_dirty(Tables T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < T.words) {
        const int rem = T.cells - i * 32;
        const unsigned m = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
        T.dirty_wire[i] = m;
        T.dirty_via[i] = m;
    }
    if (i < T.n_groups) T.group_first[i] = 0;
}

__device__ __forceinline__ Arena warp_arena(char* smem, size_t arena_b, int warp, int L, int nmax) {
    return carve_arena(smem + warp * arena_b, L, nmax);
}

// Plain DP launch: one warp per net of batch b (routes only).
__global__ void __launch_bounds__(kDpThreads) k_lshape_batch(Tables T, Plan P, int b, int stamp, int nmax,
                                                             size_t arena_b, char* gscratch, size_t gslot) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
    const int k = blockIdx.x * (blockDim.x >> 5) + warp;
    if (k >= cnt) return;
    const int id = P.ids[lo + k];
    const int N = P.node_off[id + 1] - P.node_off[id];
    Arena A;
    if (N <= nmax) A = warp_arena(smem, arena_b, warp, T.L, nmax);
    else if (gscratch) A = carve_arena(gscratch + size_t(blockIdx.x * (blockDim.x >> 5) + warp) * gslot, T.L, N);
    else { if (lane == 0) set_error(T, kELimit, id); return; }
    lshape_net(T, P, id, stamp, A, lane, false);
}

// Per-batch DP launch over every size bucket of batch b at once: CTA ranges
// [block_off[k], block_off[k+1]) serve bucket k with per_cta[k] nets per CTA
// (warps beyond it return) and an arena of nmax[k] nodes per warp (global
// scratch where nmax is 0).
struct BucketLaunch {
    int block_off[kDpBuckets + 1];
    int per[kDpBuckets];
    int nmax[kDpBuckets];
    int arena[kDpBuckets];
};
__global__ void k_lshape_bucketed(Tables T, Plan P, int b, int stamp, BucketLaunch BL, char* gscratch,
                                  size_t gslot) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int bk = 0;
    while (bk + 1 < kDpBuckets && int(blockIdx.x) >= BL.block_off[bk + 1]) ++bk;
    if (warp >= BL.per[bk]) return;
    const int lo = P.bucket_off[b * (kDpBuckets + 1) + bk], hi = P.bucket_off[b * (kDpBuckets + 1) + bk + 1];
    const int k = (int(blockIdx.x) - BL.block_off[bk]) * BL.per[bk] + warp;
    if (bk == 0) {
        // Nets of one or two nodes: 32 per warp, one per lane.
        const int q = lo + 32 * k + lane;
        lshape_net_pair(T, P, q < hi ? P.bucket_ids[q] : -1, stamp, smem + size_t(warp) * BL.arena[0], lane, false);
        return;
    }
    if (lo + k >= hi) return;
    const int id = P.bucket_ids[lo + k];
    const int N = P.node_off[id + 1] - P.node_off[id];
    const int nmax = BL.nmax[bk];
    Arena A;
    if (N <= nmax) A = warp_arena(smem, BL.arena[bk], warp, T.L, nmax);
    else if (gscratch) A = carve_arena(gscratch + size_t(k) * gslot, T.L, N);
    else { if (lane == 0) set_error(T, kELimit, id); return; }
    lshape_net(T, P, id, stamp, A, lane, false);
}

// Group each batch's nets by size bucket (one CTA per batch).
__global__ void k_plan_buckets(Plan P, int* bucket_ids, int* bucket_off) {
    __shared__ int cnt[kDpBuckets], cur[kDpBuckets];
    const int b = blockIdx.x, lo = P.batch_off[b], hi = P.batch_off[b + 1];
    if (threadIdx.x < kDpBuckets) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int k = lo + threadIdx.x; k < hi; k += blockDim.x) {
        const int id = P.ids[k];
        atomicAdd(&cnt[dp_bucket(P.node_off[id + 1] - P.node_off[id])], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = lo;
        for (int q = 0; q < kDpBuckets; ++q) {
            bucket_off[b * (kDpBuckets + 1) + q] = acc;
            cur[q] = acc;
            acc += cnt[q];
        }
        bucket_off[b * (kDpBuckets + 1) + kDpBuckets] = hi;
    }
    __syncthreads();
    for (int k = lo + threadIdx.x; k < hi; k += blockDim.x) {
        const int id = P.ids[k];
        bucket_ids[atomicAdd(&cur[dp_bucket(P.node_off[id + 1] - P.node_off[id])], 1)] = id;
    }
}

__global__ void k_commit_wires(Tables T, Plan P, int b, int stamp, int K) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
    for (int k = warp; k < cnt; k += warps) commit_net_wires(T, P, P.ids[lo + k], stamp, K, lane);
}

__global__ void k_commit_vias(Tables T, Plan P, int b, int stamp, int K) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
    commit_vias_strided(T, P, P.ids + lo, cnt, warp, warps, stamp, K, lane);
}

// refresh_cost (incremental_update.cuh:98-132) inside a persistent stage
// kernel: dirty cells (block 0 also lists the dirty groups) | prefix pass 1 |
// trees | pass 2, each phase ended by a grid barrier.  `smem`: the block's
// dynamic shared memory (per-warp pass scratch, or the tree of the group a
// block builds).  False when a barrier gave up.
__device__ __forceinline__ bool refresh_persistent(const Tables& T, GridSync& S, PhaseClock& clk, int gwarp,
                                                   int nwarps, int lane, char* smem) {
    void* xs = smem + (threadIdx.x >> 5) * prefix_xpose_bytes();
    if (blockIdx.x == 0) collect_dirty_groups(T);
    refresh_dirty_cells<2>(T, gwarp, nwarps, lane);
    if (!grid_sync(S, T)) return false;
    clk.mark(S, 4);
    const int items = *reinterpret_cast<volatile int*>(T.group_count) * T.tree_chunks;
    for (int item = gwarp; item < items; item += nwarps) {
        int g, c;
        if (prefix_item(T, item, g, c)) prefix_pass1(T, g, c, lane, xs);
    }
    if (!grid_sync(S, T)) return false;
    for (int k = blockIdx.x; k < *reinterpret_cast<volatile int*>(T.group_count); k += gridDim.x)
        prefix_tree(T, T.group_list[k], reinterpret_cast<double*>(smem));
    if (!grid_sync(S, T)) return false;
    for (int item = gwarp; item < items; item += nwarps) {
        int g, c;
        if (prefix_item(T, item, g, c)) prefix_pass2(T, g, c, lane, xs);
    }
    if (!grid_sync(S, T)) return false;
    clk.mark(S, 7);
    return true;
}

// Persistent stage: every batch of the plan in one cooperative launch.
// Per batch: recompute dirty cells (block 0 also lists the dirty prefix
// groups) -> prefix pass 1 -> prefix trees -> prefix pass 2 -> route and commit
// wires -> commit vias, separated by bounded grid barriers.
__global__ void __launch_bounds__(kPersistentThreads, 2) k_lshape_persistent(Tables T, Plan P, GridSync S,
        int stamp0, int nmax, size_t arena_b, char* gscratch, size_t gslot, int* work, DpTune tune, StageTail tail) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = warp * gridDim.x + blockIdx.x, nwarps = gridDim.x * (blockDim.x >> 5);
    PhaseClock clk;
    clk.start(S);
    for (int b = 0; b < P.n_batches; ++b) {
        const int stamp = stamp0 + b + 1;
        if (!refresh_persistent(T, S, clk, gwarp, nwarps, lane, smem)) return;
        // Route every net of the batch and commit its wires: size buckets from
        // the largest down (long nets start first), nets taken from the
        // bucket's work queue `per_grab` at a time.  (In this kernel the
        // smallest nets are the filler that evens out the warps' finish
        // times, so they too take a warp each.)
        const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
        const Arena A = warp_arena(smem, arena_b, warp, T.L, nmax);
        for (int bk = kDpBuckets - 1; bk >= 0; --bk) {
            const int blo = P.bucket_off[b * (kDpBuckets + 1) + bk], bhi = P.bucket_off[b * (kDpBuckets + 1) + bk + 1];
            const int g = tune.per_grab[bk];
            if (bk == 0 && g >= 32) {
                // Nets of one or two nodes, one per lane (lane-interleaved
                // scratch in the warp's arena), g per grab.
                while (true) {
                    int k = 0;
                    if (lane == 0) k = atomicAdd(work + b * kDpBuckets + bk, g);
                    k = __shfl_sync(0xffffffffu, k, 0);
                    if (blo + k >= bhi) break;
                    const unsigned long long t0 = S.phase_ns && lane == 0 ? global_ns() : 0ull;
                    for (int q = blo + k + lane; q < min(blo + k + g, bhi); q += 32)
                        lshape_net_pair(T, P, P.bucket_ids[q], stamp, smem + size_t(warp) * arena_b, lane, true);
                    __syncwarp();
                    if (S.phase_ns && lane == 0) {
                        const unsigned long long dt = global_ns() - t0;
                        atomicAdd(S.phase_ns + kNetTimeSlot + bk, dt);
                        atomicMax(S.phase_ns + kNetTimeSlot + kDpBuckets + bk, dt);
                    }
                }
                continue;
            }
            while (true) {
                int k = 0;
                if (lane == 0) k = atomicAdd(work + b * kDpBuckets + bk, g);
                k = __shfl_sync(0xffffffffu, k, 0);
                if (blo + k >= bhi) break;
                for (int q = blo + k; q < min(blo + k + g, bhi); ++q) {
                    const int id = P.bucket_ids[q];
                    const int N = P.node_off[id + 1] - P.node_off[id];
                    const unsigned long long t0 = S.phase_ns && lane == 0 ? global_ns() : 0ull;
                    if (N <= nmax) lshape_net(T, P, id, stamp, A, lane, true);
                    else if (gscratch) lshape_net(T, P, id, stamp, carve_arena(gscratch + size_t(gwarp) * gslot, T.L, N), lane, true);
                    else if (lane == 0) set_error(T, kELimit, id);
                    if (S.phase_ns && lane == 0) {  // profiling: warp time of every net, by size bucket
                        const unsigned long long dt = global_ns() - t0;
                        atomicAdd(S.phase_ns + kNetTimeSlot + bk, dt);
                        atomicMax(S.phase_ns + kNetTimeSlot + kDpBuckets + bk, dt);
                    }
                }
            }
        }
        if (!grid_sync(S, T)) return;
        clk.mark(S, 5);
        // Via demand sees every wire timestamp of the batch.
        commit_vias_strided(T, P, P.ids + lo, cnt, gwarp, nwarps, stamp, 1, lane);
        if (!grid_sync(S, T)) return;
        clk.mark(S, 6);
    }
    // Rip-up classification and congestion view of the final demand, in the
    // same launch (no host round trip between the stage and them).
    if (tail.flags) stage_tail_persistent(T, P, tail, S);
}

// --- FLT stage kernels (flt.cuh) --------------------------------------------
constexpr int kFltThreads = 128;

// One warp per net of batch b: layer-change tables, solve, trace, wires.
// Blocks below `nw` take the batch's wide nets, a CTA each.
__global__ void __launch_bounds__(kFltThreads) k_flt_batch(Tables T, Flt F, Plan P2, int b, int stamp, int nw) {
    const int lane = threadIdx.x & 31;
    const int lo = P2.batch_off[b], cnt = P2.batch_off[b + 1] - lo;
    if (int(blockIdx.x) < nw) {
        flt_net_block(T, F, P2, P2.ids[F.border[lo + blockIdx.x]], stamp, true);
        return;
    }
    const int k = nw + (((blockIdx.x - nw) * blockDim.x + threadIdx.x) >> 5);
    if (k < cnt) flt_net(T, F, P2, P2.ids[F.border[lo + k]], stamp, lane, true);
}

// Layer-change tables of batch b's edges (flt_edges_batch).
__global__ void k_flt_edges(Tables T, Flt F, Plan P2, int b) {
    flt_edges_batch(T, F, P2, b, (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5,
                    ((long long)gridDim.x * blockDim.x) >> 5, threadIdx.x & 31);
}

// Persistent FLT stage: per batch, [remove stage-one wires -> remove their
// vias ->] refresh cells -> prefix pass 1 -> trees -> pass 2 -> layer-change
// tables of the batch's edges -> FLT nets and wires -> vias, separated by
// bounded grid barriers (flt.cuh:141-168 order).
__global__ void __launch_bounds__(kPersistentThreads, 2) k_flt_persistent(Tables T, Flt F, Plan P1, Plan P2,
        GridSync S, int stamp0, int remove, int* work) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = warp * gridDim.x + blockIdx.x, nwarps = gridDim.x * (blockDim.x >> 5);
    PhaseClock clk;
    clk.start(S);
    for (int b = 0; b < P2.n_batches; ++b) {
        const int lo = P2.batch_off[b], cnt = P2.batch_off[b + 1] - lo;
        const int stamp = stamp0 + (remove ? 2 * b + 2 : b + 1);
        if (remove) {
            for (int k = gwarp; k < cnt; k += nwarps) commit_net_wires(T, P1, P2.ids[lo + k], stamp - 1, -1, lane);
            if (!grid_sync(S, T)) return;
            commit_vias_strided(T, P1, P2.ids + lo, cnt, gwarp, nwarps, stamp - 1, -1, lane);
            if (!grid_sync(S, T)) return;
            clk.mark(S, 6);
        }
        if (!refresh_persistent(T, S, clk, gwarp, nwarps, lane, smem)) return;
        flt_edges_batch(T, F, P2, b, gwarp, nwarps, lane);
        if (!grid_sync(S, T)) return;
        clk.mark(S, 10);
        // The batch's wide nets a CTA each, from block 0; the others a warp
        // each, to global warps in block-major order over the remaining blocks
        // (warp 0 of every block first, so a batch's nets -- often fewer than
        // the blocks -- land on different SMs, each with its L1 to itself for
        // the nets' thread-local arrays).  With at least as many wide nets as
        // blocks, every block takes wide nets in turn and then every warp the
        // others.
        const int nw = F.nwide[b], G = gridDim.x, wpb = blockDim.x >> 5;
        for (int k = blockIdx.x; k < nw; k += G) flt_net_block(T, F, P2, P2.ids[F.border[lo + k]], stamp, true);
        const int G2 = nw < G ? G - nw : G, b2 = nw < G ? int(blockIdx.x) - nw : int(blockIdx.x);
        if (b2 >= 0)
            for (int k = nw + warp * G2 + b2; k < cnt; k += G2 * wpb)
                flt_net(T, F, P2, P2.ids[F.border[lo + k]], stamp, lane, true);
        if (!grid_sync(S, T)) return;
        clk.mark(S, 5);
        commit_vias_strided(T, P2, P2.ids + lo, cnt, gwarp, nwarps, stamp, 1, lane);
        if (!grid_sync(S, T)) return;
        clk.mark(S, 6);
    }
}

// --- Z-shape stage kernels (zshape.cuh) -------------------------------------
constexpr int kZThreads = 256;
constexpr int kBoxThreads = 256;
constexpr int kMaxBoxBatch = 256;

constexpr int kZCand = 2 * (kMaxLayers + 1) * (kMaxLayers + 1);  // node-DP ranges per warp
// One CTA per net of batch b (solve<4>, zshape.cuh:62-388, with the route
// conversion of convert_routes fused into the traceback).
__global__ void __launch_bounds__(kZThreads) k_zshape_batch(Tables T, ZTrees Z, Plan P, int b) {
    __shared__ int cand[kZCand];
    const int lo = P.batch_off[b];
    zshape_net(T, Z, P, P.ids[lo + blockIdx.x], 0, threadIdx.x, blockDim.x, false, cand);
}
// Thread-per-net commit (commit_wire_demand / commit_via_demand,
// demand.cuh:129-232), the Z-shape pipeline's form (pipeline_ggr.hpp:132-133).
__global__ void k_commit_thread_wires(Tables T, Plan P, int b, int stamp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
    if (i < cnt) commit_thread_wires(T, P, P.ids[lo + i], stamp, 1);
}
__global__ void k_commit_thread_vias(Tables T, Plan P, int b, int stamp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
    if (i < cnt) commit_thread_vias(T, P, P.ids[lo + i], stamp, 1);
}

// Persistent Z-shape stage: per batch, refresh cells -> prefix pass 1 ->
// trees -> pass 2 -> Z-shape nets and their wires -> vias.
__global__ void __launch_bounds__(kPersistentThreads, 2) k_zshape_persistent(Tables T, ZTrees Z, Plan P, GridSync S,
                                                                              int stamp0, int* work) {
    extern __shared__ __align__(16) char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = warp * gridDim.x + blockIdx.x, nwarps = gridDim.x * (blockDim.x >> 5);
    __shared__ int cand[kZCand];
    __shared__ int znet;
    PhaseClock clk;
    clk.start(S);
    for (int b = 0; b < P.n_batches; ++b) {
        const int lo = P.batch_off[b], cnt = P.batch_off[b + 1] - lo;
        const int stamp = stamp0 + b + 1;
        if (!refresh_persistent(T, S, clk, gwarp, nwarps, lane, smem)) return;
        while (true) {  // one CTA per net
            if (threadIdx.x == 0) znet = atomicAdd(work + b, 1);
            __syncthreads();
            const int k = znet;
            __syncthreads();
            if (k >= cnt) break;
            zshape_net(T, Z, P, P.ids[lo + k], stamp, threadIdx.x, blockDim.x, true, cand);
        }
        if (!grid_sync(S, T)) return;
        clk.mark(S, 5);
        commit_vias_strided(T, P, P.ids + lo, cnt, gwarp, nwarps, stamp, 1, lane);
        if (!grid_sync(S, T)) return;
        clk.mark(S, 6);
    }
}

// Bounding-box refinement of every group (current plan batch) at once, one
// CTA per group: keys (area, id) merge-sorted descending by the CTA, then
// warp 0 forms the greedy rounds (zshape_topology.hpp:7-57) with the round's
// boxes in shared memory, 32 pending nets fetched per memory round trip.
// Writes the rounds in order into tmp (the group's own id range), their sizes
// into bsize and their number into rounds[g].
__global__ void __launch_bounds__(kBoxThreads) k_bbox_refine(const int* ids, const int* batch_off, const int4* box,
        unsigned long long* ka, unsigned long long* kb, int* pend, int* tmp, int* bsize, int* rounds, int max_batch) {
    __shared__ int4 rect[kMaxBoxBatch];
    const int g = blockIdx.x, tid = threadIdx.x;
    const int lo = batch_off[g], n = batch_off[g + 1] - lo;
    for (int k = tid; k < n; k += blockDim.x) {
        const int id = ids[lo + k];
        const int4 bb = box[id];
        const unsigned long long area = static_cast<unsigned long long>(bb.y - bb.x + 1) * (bb.w - bb.z + 1);
        ka[lo + k] = (area << 32) | static_cast<unsigned>(id);
    }
    __syncthreads();
    unsigned long long* src = ka + lo;
    unsigned long long* dst = kb + lo;
    for (int w = 1; w < n; w <<= 1) {
        for (int k = tid; k < n; k += blockDim.x) {
            const int start = (k / (2 * w)) * (2 * w), mid = min(start + w, n), end = min(start + 2 * w, n);
            const unsigned long long key = src[k];
            int a = k < mid ? mid : start, e = k < mid ? end : mid;
            const int base = k < mid ? k - start : k - mid;
            const int first = a;
            while (a < e) {  // elements of the other run that sort before `key` (keys are distinct)
                const int m = (a + e) >> 1;
                if (src[m] > key) a = m + 1;
                else e = m;
            }
            dst[start + base + (a - first)] = key;
        }
        __syncthreads();
        unsigned long long* t = src; src = dst; dst = t;
    }
    for (int k = tid; k < n; k += blockDim.x) pend[lo + k] = static_cast<int>(src[k] & 0xffffffffu);
    __syncthreads();
    if (tid >= 32) return;
    const int lane = tid;
    int remaining = n, r = 0, out = 0;
    while (remaining > 0) {
        int count = 0;
        bool full = false;
        for (int base = 0; base < remaining && !full; base += 32) {
            const int myid = base + lane < remaining ? pend[lo + base + lane] : -1;
            const int4 mb = myid >= 0 ? box[myid] : make_int4(0, -1, 0, -1);
            const int lim = min(32, remaining - base);
            for (int q = 0; q < lim; ++q) {
                const int id = __shfl_sync(0xffffffffu, myid, q);
                int4 bb;
                bb.x = __shfl_sync(0xffffffffu, mb.x, q);
                bb.y = __shfl_sync(0xffffffffu, mb.y, q);
                bb.z = __shfl_sync(0xffffffffu, mb.z, q);
                bb.w = __shfl_sync(0xffffffffu, mb.w, q);
                bool hit = false;
                for (int m = lane; m < count; m += 32) hit |= boxes_meet(rect[m], bb);
                if (__any_sync(0xffffffffu, hit)) continue;
                if (lane == 0) {
                    rect[count] = bb;
                    tmp[lo + out] = id;
                    pend[lo + base + q] = -1;
                }
                __syncwarp();
                ++count;
                ++out;
                if (count == max_batch) { full = true; break; }
            }
        }
        if (lane == 0) bsize[lo + r] = count;
        ++r;
        __syncwarp();
        // Stable in-place compaction of the nets still pending.
        int kept = 0;
        for (int base = 0; base < remaining; base += 32) {
            const int v = base + lane < remaining ? pend[lo + base + lane] : -1;
            const unsigned keep = __ballot_sync(0xffffffffu, v >= 0);
            __syncwarp();
            if (v >= 0) pend[lo + kept + __popc(keep & ((1u << lane) - 1u))] = v;
            kept += __popc(keep);
            __syncwarp();
        }
        remaining = kept;
    }
    if (lane == 0) rounds[g] = r;
}

// Lay the rounds of group g out in reverse order (the stage runs the refined
// batch list reversed, pipeline_ggr.hpp:55): ids and new batch offsets.
__global__ void k_bbox_scatter(const int* batch_off, const int* tmp, const int* bsize, const int* rounds,
                               const int* first_batch, int* bofs, int* ids_out, int* off_out) {
    const int g = blockIdx.x, tid = threadIdx.x;
    const int lo = batch_off[g], n = batch_off[g + 1] - lo, R = rounds[g], B = first_batch[g];
    if (tid == 0) {
        int o = 0;
        for (int r = 0; r < R; ++r) {
            bofs[lo + r] = o;
            off_out[B + (R - 1 - r)] = lo + n - o - bsize[lo + r];
            o += bsize[lo + r];
        }
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < R; r += nw) {
        const int o = bofs[lo + r], sz = bsize[lo + r];
        const int dst = lo + n - o - sz;
        for (int k = lane; k < sz; k += 32) ids_out[dst + k] = tmp[lo + o + k];
    }
}

// --- soft-min DAG and adjoint (softmin.cuh) ---------------------------------
constexpr int kSoftThreads = 128;

template <class T>
__global__ void k_soft_tables(Tables Tb, Soft<T> S) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < Tb.cells) soft_tables_cell<T>(Tb, S, c);
}
// Track k of layer l (one thread each): first cell, stride and length.
__device__ __forceinline__ bool soft_track(const Tables& Tb, int t, int& base, int& stride, int& len) {
    const int M = max(Tb.X, Tb.Y), l = t / M, k = t - l * M;
    if (l >= Tb.L) return false;
    if (along_y(Tb, l)) {
        if (k >= Tb.X) return false;
        base = cell_index(Tb, l, k, 0); stride = 1; len = Tb.Y;
    } else {
        if (k >= Tb.Y) return false;
        base = cell_index(Tb, l, 0, k); stride = Tb.Y; len = Tb.X;
    }
    return true;
}
template <class T>
__global__ void k_soft_prefix(Tables Tb, Soft<T> S) {
    int base, stride, len;
    if (!soft_track(Tb, blockIdx.x * blockDim.x + threadIdx.x, base, stride, len)) return;
    T acc = 0;
    for (int q = 0; q < len; ++q) {
        S.P[base + q * stride] = acc;
        acc += S.wc[base + q * stride];
    }
}
// One thread per net; a net's range tables (and their adjoints) sit in the
// scratch at twice its first node's index times L*L, so every net of the
// design runs at once.
template <class T>
__global__ void __launch_bounds__(kSoftThreads) k_soft_forward(Tables Tb, Soft<T> S, Plan P, int n) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    T* dist = S.slot + size_t(2) * P.node_off[id] * Tb.L * Tb.L;
    S.net_cost[id] = P.node_off[id + 1] > P.node_off[id] ? soft_net_forward<T>(Tb, S, P, id, dist) : T(0);
}
template <class T>
__global__ void __launch_bounds__(kSoftThreads) k_soft_backward(Tables Tb, Soft<T> S, Plan P, int n, T g) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int N = P.node_off[id + 1] - P.node_off[id];
    T* dist = S.slot + size_t(2) * P.node_off[id] * Tb.L * Tb.L;
    T* gd = dist + size_t(N) * Tb.L * Tb.L;
    if (N > 0) soft_net_backward<T>(Tb, S, P, id, dist, gd, g);
}
// dwc[j] = sum over later track positions of dP (presum[i] = sum_{j<i} wc[j]).
template <class T>
__global__ void k_soft_suffix(Tables Tb, Soft<T> S, T* dwc) {
    int base, stride, len;
    if (!soft_track(Tb, blockIdx.x * blockDim.x + threadIdx.x, base, stride, len)) return;
    T acc = 0;
    for (int q = len - 1; q >= 0; --q) {
        dwc[base + q * stride] = acc;
        acc += S.dP[base + q * stride];
    }
}
// Chain rule to capacity and the per-edge unit wire cost.
template <class T>
__global__ void k_soft_chain(Tables Tb, Soft<T> S, const T* dwc, T* dcap, T* duw) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Tb.cells) return;
    const int l = c / Tb.XY, rem = c - l * Tb.XY, x = rem / Tb.Y, y = rem - x * Tb.Y;
    const bool ay = along_y(Tb, l);
    const int pos = ay ? y : x, len = ay ? Tb.Y : Tb.X, stride = ay ? 1 : Tb.Y;
    T g = dwc[c] * soft_incr_dcap<T>(Tb, S, c, l, 1);
    if (pos == 0) g += S.dvc[c] * soft_incr_dcap<T>(Tb, S, c, l, 1);
    else if (pos < len - 1) g += S.dvc[c] * soft_incr_dcap<T>(Tb, S, c, l, static_cast<T>(0.5));
    if (pos + 1 == len - 1) g += S.dvc[c + stride] * soft_incr_dcap<T>(Tb, S, c, l, 1);
    else if (pos + 1 < len - 1) g += S.dvc[c + stride] * soft_incr_dcap<T>(Tb, S, c, l, static_cast<T>(0.5));
    dcap[c] = g;
    duw[c] = dwc[c] * static_cast<T>(soft_edge_len(Tb, l, x, y));
}
// Deterministic sum of v[0..n) into *out (one CTA).
template <class T>
__global__ void __launch_bounds__(1024) k_soft_sum(const T* v, int n, double* out) {
    __shared__ double part[1024];
    double acc = 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) acc += static_cast<double>(v[k]);
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

// --- input validation ------------------------------------------------------
// Every index a stage kernel will dereference is checked on the device after
// the upload (one thread per net, then one per geometry element); the first
// violation is recorded as (code, item) and the largest tree size kept.
struct NetCheck {
    const int* node_off; const int* nodes; const int* parents; const long long* route_off;
    const int* point_off; const int* points; const int* hseg_off; const int* hsegs;
    const int* vseg_off; const int* vsegs;
    int n, nn, np, nh, nv, XY, L;
    long long rw;
    int* status;  // [0] code (1 offsets, 2 node, 3 parent, 4 geometry), [1] item, [2] max nodes
};
__device__ __forceinline__ void check_fail(const NetCheck& C, int code, int item) {
    if (atomicCAS(C.status, 0, code) == 0) C.status[1] = item;
}
__global__ void k_validate_nets(NetCheck C) {
    const int nt = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += nt) {
        const int a = C.node_off[i], b = C.node_off[i + 1];
        const bool geo = (C.point_off[i] <= C.point_off[i + 1] && C.point_off[i] >= 0 && C.point_off[i + 1] <= C.np) &&
                         (C.hseg_off[i] <= C.hseg_off[i + 1] && C.hseg_off[i] >= 0 && C.hseg_off[i + 1] <= C.nh) &&
                         (C.vseg_off[i] <= C.vseg_off[i + 1] && C.vseg_off[i] >= 0 && C.vseg_off[i + 1] <= C.nv);
        if (a < 0 || b < a || b > C.nn || C.route_off[i] < 0 || C.route_off[i + 1] < C.route_off[i] ||
            C.route_off[i + 1] > C.rw || !geo) {
            check_fail(C, 1, i);
            continue;
        }
        atomicMax(C.status + 2, b - a);
        for (int k = a; k < b; ++k) {
            const int v = C.nodes[k], p = C.parents[k];
            if (v < 0 || v / C.XY > C.L) { check_fail(C, 2, i); break; }
            if (k == a ? p != -1 : (p < 0 || p >= k - a)) { check_fail(C, 3, i); break; }
        }
    }
    const long long total = (long long)C.np + 2ll * C.nh + 2ll * C.nv;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += nt) {
        const int v = k < C.np ? C.points[k] : k < C.np + 2ll * C.nh ? C.hsegs[k - C.np] : C.vsegs[k - C.np - 2ll * C.nh];
        if (v < 0 || v >= C.XY) check_fail(C, 4, int(k));
    }
}

// --- topology construction (topology.cuh) -----------------------------------
__global__ void k_topo_count(TopoBuild B) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < B.n) topo_count(B, id);
}
__global__ void k_topo_fill(TopoBuild B) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < B.n) topo_fill(B, id);
}

// --- maze stage (maze.cuh) ---------------------------------------------------
struct RemoveList {
    const int* ids;
    const unsigned char* phase2;
    int n;
};
__global__ void k_maze_remove(Tables T, Plan P, Plan P2, RemoveList R) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R.n) return;
    const int id = R.ids[k];
    maze_remove_route(T, R.phase2[k] ? P2.routes + P2.route_off[id] : P.routes + P.route_off[id]);
}
__global__ void __launch_bounds__(kScoreThreads) k_maze_score(Tables T, double* partials) { maze_score_partial(T, partials); }

// --- .out text (outfmt.cuh): one warp per record ---------------------------
__global__ void k_out_count(OutRecords R) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r < R.n) out_count(R, r, threadIdx.x & 31);
}
__global__ void k_out_write(OutRecords R) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r < R.n) out_write(R, r, threadIdx.x & 31);
}

// --- batching kernels -------------------------------------------------------
// Flat lists: per-position counts (warp per position), exclusive scans, fill.
__global__ void k_flat_count(BatchState B, int n_nets) {
    const int warps = gridDim.x * blockDim.x / 32;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) / 32; p < B.n; p += warps) {
        const int id = B.order[p];
        if (id < 0 || id >= n_nets) {  // refused on the host after the scan
            if ((threadIdx.x & 31) == 0) { batch_error(B, kEInval, p); B.mark_off[p] = 0; B.pt_off[p] = 0; }
            continue;
        }
        flat_count(B, p);
    }
}
__global__ void k_flat_fill(BatchState B) {
    const int warps = gridDim.x * blockDim.x / 32;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) / 32; p < B.n; p += warps) flat_fill(B, p);
}

// Exclusive scan of a[0..n) in place with the total at a[n]: tiles of
// kScanTile, a scan of the tile totals, then the tile offsets added.
constexpr int kScanTile = 1024;  // 256 threads x 4 elements
__device__ __forceinline__ long long block_incl_scan(long long v, long long* ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) ws[warp] = v;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < nw ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        if (lane < nw) ws[lane] = w;
    }
    __syncthreads();
    const long long r = v + (warp ? ws[warp - 1] : 0);
    __syncthreads();  // ws is reused by the next call
    return r;
}
__global__ void __launch_bounds__(256) k_scan_tiles(long long* a, int n, long long* sums) {
    __shared__ long long ws[32];
    const long long base = blockIdx.x * (long long)kScanTile + threadIdx.x * 4;
    long long v[4], t = 0;
    for (int k = 0; k < 4; ++k) {
        v[k] = base + k < n ? a[base + k] : 0;
        t += v[k];
    }
    long long run = block_incl_scan(t, ws) - t;
    for (int k = 0; k < 4; ++k) {
        if (base + k < n) a[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = run;
}
__global__ void __launch_bounds__(1024) k_scan_sums(long long* sums, int tiles) {
    __shared__ long long ws[32];
    __shared__ long long total;
    long long carry = 0;
    for (int base = 0; base < tiles; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const long long v = i < tiles ? sums[i] : 0;
        const long long incl = block_incl_scan(v, ws);
        if (i < tiles) sums[i] = carry + incl - v;
        if (threadIdx.x == blockDim.x - 1) total = incl;
        __syncthreads();
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[tiles] = carry;
}
__global__ void k_scan_add(long long* a, int n, const long long* sums, int tiles) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) a[i] += sums[i / kScanTile];
    if (i == 0) a[n] = sums[tiles];
}

// Route words in use per net: the count word and the words below it,
// clamped to the net's storage (at least the count word).
__global__ void k_route_used(const int* routes, const long long* route_off, int n, long long* used) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long cap = route_off[i + 1] - route_off[i];
    used[i] = cap > 0 ? max(1ll, min(static_cast<long long>(routes[route_off[i]]), cap)) : 0;
}
// One warp per net moves its words in use between the route storage and a
// packed array (pos: exclusive prefix of the words in use).
__global__ void k_route_move(const long long* route_off, const long long* pos, int n, int* routes, int* packed,
                             int to_packed) {
    const int lane = threadIdx.x & 31;
    for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((long long)gridDim.x * blockDim.x) >> 5) {
        const long long a = pos[i], m = pos[i + 1] - a, r = route_off[i];
        for (long long k = lane; k < m; k += 32) {
            if (to_packed) packed[a + k] = routes[r + k];
            else routes[r + k] = packed[a + k];
        }
    }
}

// Plain form: one launch per step and chunk.
__device__ __forceinline__ long long launch_thread() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long launch_threads() { return (long long)gridDim.x * blockDim.x; }
template <int CH>
__global__ void k_batch_point_bits(BatchState B, int s) { batch_point_bits<CH>(B, s, true, launch_thread(), launch_threads()); }
template <int CH>
__global__ void k_batch_raster(BatchState B, int s) { batch_raster<CH>(B, s, 0, launch_thread(), launch_threads()); }
template <int CH>
__global__ void k_batch_gather(BatchState B, int s) {
    batch_gather<CH>(B, s, 0, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}
template <int CH>
__global__ void __launch_bounds__(CH) k_batch_solve(BatchState B, int s) {
    extern __shared__ __align__(16) unsigned bsm[];
    if (*reinterpret_cast<volatile int*>(B.error)) return;
    const SolveSmem S = solve_smem<CH>(bsm, B.W);
    const int C = 32 * B.W;
    for (int k = threadIdx.x; k < C; k += blockDim.x) S.cnt[k] = B.count[k];
    if (S.per_warp)
        for (int k = threadIdx.x; k < (CH / 32) * C; k += blockDim.x) S.wh[k] = 0;
    for (int k = threadIdx.x; k < B.W; k += blockDim.x) S.full[k] = B.fullmask[k];
    __syncthreads();
    if (!batch_solve<CH>(B, s, false, S)) return;
    for (int k = threadIdx.x; k < C; k += blockDim.x) B.count[k] = S.cnt[k];
    for (int k = threadIdx.x; k < B.W; k += blockDim.x) B.fullmask[k] = S.full[k];
}
// Publish chunk s, empty its chunk-local mask and query-point bits, and set
// the next chunk's query-point bits.
template <int CH>
__global__ void k_batch_publish(BatchState B, int s) {
    if (*reinterpret_cast<volatile int*>(B.error)) return;
    const long long t = launch_thread(), nt = launch_threads();
    batch_publish<CH>(B, s, t, nt);
    batch_clear<CH>(B, s, 0, t, nt);
    batch_point_bits<CH>(B, s, false, t, nt);
    if (s + CH < B.n) batch_point_bits<CH>(B, s + CH, true, t, nt);
}

// Persistent batching: CTAs of kPersistThreads threads, one per SM, at least
// two.  CTA 0 is the solver and has its SM to itself (its first CH
// threads solve, the rest leave): for chunk r it waits until the other CTAs
// (G of them, one shared barrier counter) have gathered chunk r, solves it,
// and releases `solved` = r + 1.  The other CTAs set the query-point bits of
// chunks 0-4 | raster chunks 0 and 1 | gather chunk 0 | and then run, per
// round r, one phase and one barrier:
//   wait for chunk r-1's colours; publish chunk r-1 and clear its query-point
//   bits; empty chunk r-2's chunk-local mask; set the query-point bits of
//   chunk r+5; gather chunk r+1 (cellmask as of chunk r-2 at least, chunk r-1
//   through its chunk-local mask and its colours, chunk r through the
//   previous-chunk bits the solver resolves); raster chunk r+2, keeping the
//   marks on query points of chunks r+2 to r+4              | barrier
// A chunk's local mask (five buffers, chunk k in buffer k % 5) is written by
// its raster in round k-2, read by the gathers of chunks k, k+1 and k+2
// (rounds k-1 to k+1) and emptied in round k+2, before the raster of chunk
// k+5 in round k+3.  The barrier of round r is what the solver waits for
// before chunk r+1 (counter (3 + (r + 1)) * G).
constexpr int kPersistThreads = kChunkMax;
template <int CH>
__global__ void __launch_bounds__(kPersistThreads, 1) k_batch_persistent(BatchState B, GridSync S, Tables T) {
    extern __shared__ __align__(16) unsigned bsm[];
    __shared__ int go;
    const int chunks = (B.n + CH - 1) / CH;
    const unsigned G = gridDim.x - 1;
    if (blockIdx.x == 0) {
        if (threadIdx.x >= CH) return;
        PhaseClock clk{0, 0};
        clk.start(S);
        const SolveSmem M = solve_smem<CH>(bsm, B.W);
        const int C = 32 * B.W;
        for (int k = threadIdx.x; k < C; k += CH) M.cnt[k] = B.count[k];
        if (M.per_warp)
            for (int k = threadIdx.x; k < (CH / 32) * C; k += CH) M.wh[k] = 0;
        for (int k = threadIdx.x; k < B.W; k += CH) M.full[k] = B.fullmask[k];
        for (int r = 0; r < chunks; ++r) {
            if (threadIdx.x == 0) go = wait_at_least(S.count, (3u + unsigned(r)) * G, S.timeout_ns, T, true);
            solve_sync<CH>();
            if (!go) return;
            clk.mark(S, 8);
            if (!batch_solve<CH>(B, r * CH, r > 0, M)) return;
            __threadfence();
            solve_sync<CH>();
            if (threadIdx.x == 0) asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(B.solved), "r"(unsigned(r + 1)) : "memory");
            clk.mark(S, 2);
        }
        for (int k = threadIdx.x; k < C; k += CH) B.count[k] = M.cnt[k];
        for (int k = threadIdx.x; k < B.W; k += CH) B.fullmask[k] = M.full[k];
        return;
    }
    PhaseClock clk{0, 1};
    clk.start(S);
    const long long t = (blockIdx.x - 1) * (long long)blockDim.x + threadIdx.x, nt = (long long)G * blockDim.x;
    for (int k = 0; k < 5 && k < chunks; ++k) batch_point_bits<CH>(B, k * CH, true, t, nt);
    if (!grid_sync_of(S, T, G)) return;
    for (int k = 0; k < 2 && k < chunks; ++k) batch_raster<CH>(B, k * CH, 2, t, nt);
    if (!grid_sync_of(S, T, G)) return;
    batch_gather<CH>(B, 0, 0, t, nt);
    if (!grid_sync_of(S, T, G)) return;
    clk.mark(S, 1);
    for (int r = 0; r < chunks; ++r) {
        if (r >= 1) {
            if (threadIdx.x == 0) go = wait_at_least(B.solved, unsigned(r), S.timeout_ns, T, true);
            __syncthreads();
            if (!go) return;
            clk.mark(S, 9);
            batch_publish<CH>(B, (r - 1) * CH, t, nt);
            batch_point_bits<CH>(B, (r - 1) * CH, false, t, nt);
        }
        if (r >= 2) batch_clear<CH>(B, (r - 2) * CH, 2, t, nt);
        if (r + 5 < chunks) batch_point_bits<CH>(B, (r + 5) * CH, true, t, nt);
        if (r + 1 < chunks) batch_gather<CH>(B, (r + 1) * CH, min(r + 1, 2), t, nt);
        if (r + 2 < chunks) batch_raster<CH>(B, (r + 2) * CH, 2, t, nt);
        if (!grid_sync_of(S, T, G)) return;
        clk.mark(S, 1);
    }
    if (chunks > 0) {
        if (threadIdx.x == 0) go = wait_at_least(B.solved, unsigned(chunks), S.timeout_ns, T, true);
        __syncthreads();
        if (!go) return;
        batch_publish<CH>(B, (chunks - 1) * CH, t, nt);
        batch_point_bits<CH>(B, (chunks - 1) * CH, false, t, nt);
        for (int k = max(chunks - 2, 0); k < chunks; ++k) batch_clear<CH>(B, k * CH, 2, t, nt);
    }
}

// Position of every net inside its batch: the number of earlier order
// positions with the same colour.  A stable counting pass over tiles of
// kRankTile positions: per-tile colour counts, their exclusive scan per
// colour over the tiles, then the ranks inside each tile (warps in turn).
constexpr int kRankTile = 1024;
__global__ void __launch_bounds__(kRankTile) k_rank_counts(const int* batch_of, int n, int C, int* tile_cnt) {
    extern __shared__ int hist[];  // [C]
    for (int k = threadIdx.x; k < C; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const long long p = blockIdx.x * (long long)kRankTile + threadIdx.x;
    if (p < n) atomicAdd(hist + batch_of[p], 1);
    __syncthreads();
    for (int k = threadIdx.x; k < C; k += blockDim.x) tile_cnt[size_t(blockIdx.x) * C + k] = hist[k];
}
__global__ void k_rank_scan(int* tile_cnt, int tiles, int C) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    int acc = 0;
    for (int t = 0; t < tiles; ++t) {
        const int v = tile_cnt[size_t(t) * C + c];
        tile_cnt[size_t(t) * C + c] = acc;
        acc += v;
    }
}
__global__ void __launch_bounds__(kRankTile) k_rank_assign(const int* batch_of, int n, int C, const int* tile_base,
                                                           int* rank) {
    extern __shared__ int run[];  // [C] counts of the tile's earlier warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < C; k += blockDim.x) run[k] = 0;
    __syncthreads();
    const long long p = blockIdx.x * (long long)kRankTile + threadIdx.x;
    const int c = p < n ? batch_of[p] : -1 - lane;  // distinct dummies for idle lanes
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int within = __popc(peers & ((1u << lane) - 1u));
    const bool leader = p < n && lane == __ffs(peers) - 1;
    for (int w = 0; w < kRankTile / 32; ++w) {
        if (warp == w) {
            if (p < n) rank[p] = tile_base[size_t(blockIdx.x) * C + c] + run[c] + within;
            __syncwarp();
            if (leader) run[c] += __popc(peers);
        }
        __syncthreads();
    }
}

// Batch offsets in execution order (reversed colours) and the flattened ids.
__global__ void k_plan_offsets(BatchState B, int* batch_off) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nb = *B.n_colors;
    batch_off[0] = 0;
    for (int e = 0; e < nb; ++e) batch_off[e + 1] = batch_off[e] + B.count[nb - 1 - e];
}
__global__ void k_plan_scatter(BatchState B, const int* batch_off, int* ids) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.n) return;
    const int nb = *B.n_colors, c = B.batch_of[j];
    ids[batch_off[nb - 1 - c] + B.rank[j]] = B.order[j];
}

// --- rip-up classification and congestion view -----------------------------
// Rip-up classification and congestion view (device/congestion.cuh).
__global__ void k_mark_overflow(Tables T, int threshold, int* of_sum) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < T.cells) overflow_mark(T, threshold, of_sum, c);
}
__global__ void k_int_prefix(Tables T, int* v) { overflow_prefix_track(T, v, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_overflow_nets(Tables T, Plan P, int n, const int* of_sum, unsigned char* is_of) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < n) overflow_net(T, P, of_sum, is_of, id);
}
// The same with each net's current route: phase two where phase2[id] is set
// (mark_overflow_nets, congestion.cuh:30-45).
__global__ void k_overflow_nets2(Tables T, Plan P, Plan P2, int n, const int* of_sum, const unsigned char* phase2,
                                 unsigned char* is_of) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const Plan& Q = phase2[id] ? P2 : P;
    is_of[id] = overflow_route(T, Q.routes + Q.route_off[id], Q.route_off[id + 1] > Q.route_off[id], of_sum);
}
__global__ void k_congestion(Tables T, unsigned char* cong, float* xsum, float* ysum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < T.XY) congestion_cell(T, cong, xsum, ysum, i);
}
__global__ void k_float_line_prefix(float* v, int lines, int len, int line_stride, int elem_stride) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < lines) congestion_line_prefix(v + size_t(t) * line_stride, len, elem_stride);
}

// Cost-term table (Tables::of_table): entry ((l, k), h) = the terms of a
// cell of capacity caps[k] and demand h half-units on layer l, by the same
// functions the kernels would evaluate.
constexpr int kOfDmax = 512;  // demands below 512 half-units come from the table
__global__ void k_build_of_table(Tables T, const float* caps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.L * T.of_rows * T.of_stride) return;
    const int row = i / T.of_stride, h = i - row * T.of_stride;
    const int l = row / T.of_rows, k = row - l * T.of_rows;
    double one, half;
    cell_terms(T, caps[k], h, T.short_costs[l], one, half);
    const_cast<double2*>(T.of_table)[i] = terms_of(one, half);
}

// The cost model's exponential for n values (grb_cost_exp).
__global__ void k_cost_exp(const float* x, int n, float* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = cost_exp(x[i]);
}

}  // namespace

// ---------------------------------------------------------------------------
// Fixed scratch for grb_ripup_classify_noalloc
// ---------------------------------------------------------------------------
// The rip-up classification needs one int per grid cell (overflow marks, then
// their prefix along each track) and one flag per net.  For callers that must
// not allocate device memory this scratch lives in one file-scope array that
// every GPU loading the library holds until the process exits:
// (4,194,304 + 262,144) ints = 17,825,792 bytes = 17.0 MiB.
constexpr int kNoAllocCells = 4 << 20;  // at most 4,194,304 grid cells (L*X*Y)
constexpr int kNoAllocNets = 1 << 20;   // at most 1,048,576 nets
constexpr int kNoAllocWords = kNoAllocCells + kNoAllocNets / 4;
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocWords];

// ---------------------------------------------------------------------------
// Host context
// ---------------------------------------------------------------------------
struct grb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 0;
    std::string error;
    Tables T{};
    std::vector<void*> owned;
    int stamp = 0;
    int64_t launches = 0;
    // net store
    int n_nets = 0;
    int max_nodes = 0;
    long long route_words = 0;
    int *node_off = nullptr, *nodes = nullptr, *parents = nullptr;
    long long* route_off = nullptr;
    int* routes = nullptr;
    int *point_off = nullptr, *points = nullptr, *hseg_off = nullptr, *hsegs = nullptr, *vseg_off = nullptr, *vsegs = nullptr;
    std::vector<void*> net_bufs;
    long long net_cap[6] = {0, 0, 0, 0, 0, 0};  // nets, nodes, route words, points, hsegs, vsegs
    // plan
    int *ids = nullptr, *batch_off = nullptr;
    int plan_n = 0, n_batches = 0, plan_cap = 0;
    std::vector<int> h_batch_off;
    int plan_version = 0;
    // scratch
    char* gscratch = nullptr;
    size_t gscratch_bytes = 0;
    int* work = nullptr;
    int work_cap = 0;
    unsigned* sync = nullptr;   // [count, generation]
    // batching buffers
    unsigned *cellmask = nullptr, *fmask = nullptr, *fullmask = nullptr;
    unsigned* lmask[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // chunk-local masks
    unsigned* ptchunk = nullptr;                        // [X*Y] query-point bits by chunk % 32
    unsigned *pred = nullptr, *prevp = nullptr, *bsolved = nullptr;
    bool lmask_dirty = false;          // a run stopped before clearing them
    int *bcount = nullptr, *ncolors = nullptr, *batch_of = nullptr, *brank = nullptr, *order = nullptr;
    int* rank_tiles = nullptr;         // [tiles][colours] scratch of the rank pass
    size_t rank_cap = 0;
    int bW = 0, bn_cap = 0;
    // flat mark / query-point lists by order position
    long long *mark_off = nullptr, *pt_off = nullptr, *scan_sums = nullptr;
    unsigned *mark_cell = nullptr, *pt_cell = nullptr;
    unsigned short *mark_jj = nullptr, *pt_jj = nullptr;
    long long mark_cap = 0, pt_cap = 0;
    // FLT stage (grb_upload_geometry / grb_upload_flt)
    std::vector<void*> geom_bufs;     // batching geometry replacing the uploaded one
    std::vector<void*> flt_bufs;
    std::vector<void*> topo_bufs;     // grb_build_topology: uploaded trees, counts, DFS stack
    // maze stage (grb_remove_routes, grb_routing_score, grb_checkpoint)
    int* ckpt_demand = nullptr;       // demand snapshot
    double ckpt_wirelength = 0;
    unsigned long long ckpt_vias = 0;
    double* score_partials = nullptr;
    // .out text (grb_format_out / grb_drain_out)
    std::vector<void*> out_bufs;      // uploaded records and per-record byte offsets
    char* out_text = nullptr;
    long long out_text_cap = 0, out_bytes = 0;
    bool out_pending = false;         // formatted text not yet drained
    cudaStream_t out_stream = nullptr;
    cudaEvent_t out_ready = nullptr, out_chunk_ev[2] = {nullptr, nullptr};
    char* out_host[2] = {nullptr, nullptr};  // pinned chunk buffers
    long long topo_sizes[4] = {-1, 0, 0, 0};  // nodes, points, h-, v-segments of the net store (-1: none)
    Flt F{};
    long long route2_words = 0;
    int flt_n = -1;                   // nets covered by the uploaded DAGs
    std::vector<int> h_flt_node_off;
    std::vector<int> h_flt_edge_off;
    int* flt_eprefix = nullptr;       // [plan+1] first edge slot of each plan position
    int* flt_emap = nullptr;          // plan position of each edge slot
    long long flt_emap_cap = 0;
    int flt_emap_plan = -1, flt_emap_flt = -1;  // plan / DAG versions the map was built for
    std::vector<long long> h_route2_off;
    std::vector<void*> used_bufs;     // grb_read/write_routes_used: positions, tile sums, packed words
    long long used_n_cap = -1, used_words_cap = 0;
    long long* used_pos = nullptr;
    long long* used_sums = nullptr;
    int* used_pack = nullptr;
    std::vector<int> h_flt_width;     // per net: nodes of its widest DAG level
    int flt_block_width = 32;         // wider nets are routed by a whole CTA (< 0: none)
    int* flt_border = nullptr;        // plan positions, each batch's wide nets first
    int* flt_nwide = nullptr;         // wide nets per batch
    long long flt_border_cap = 0, flt_nwide_cap = 0;
    long long flt_border_key[3] = {-1, -1, -1};  // plan, DAG versions and width it was built for
    std::vector<int> h_flt_nwide;
    int flt_version = 0;
    cudaGraphExec_t flt_graph = nullptr;
    long long flt_graph_key[5] = {-1, -1, -1, -1, -1};
    int64_t flt_graph_kernels = 0;
    // Z-shape stage (grb_upload_zshape)
    std::vector<void*> z_bufs;
    ZTrees Z{};
    int4* z_box = nullptr;            // per net (minx, maxx, miny, maxy)
    // bounding-box refinement scratch (grb_plan_bbox_batches), grow-only
    std::vector<void*> box_bufs;
    unsigned long long *box_ka = nullptr, *box_kb = nullptr;
    int *box_pend = nullptr, *box_tmp = nullptr, *box_bsize = nullptr, *box_bofs = nullptr;
    int *box_rounds = nullptr, *box_first = nullptr, *box_off = nullptr;
    int box_cap_n = 0, box_cap_g = 0;
    int z_n = -1;
    std::vector<int> h_z_node_off;
    int z_version = 0;
    cudaGraphExec_t z_graph = nullptr;
    long long z_graph_key[3] = {-1, -1, -1};
    int64_t z_graph_kernels = 0;
    // soft-min workspace (grb_softmin_forward / backward)
    std::vector<void*> soft_bufs;
    char* soft_cells = nullptr;       // 6 arrays of cells doubles
    char* soft_slot = nullptr;
    size_t soft_slot_bytes = 0;
    double* soft_scalar = nullptr;
    int* check = nullptr;             // [3] upload validation status
    // size-bucketed plan and tuned launch shapes
    int* bucket_ids = nullptr;
    int* bucket_off = nullptr;
    int bucket_cap = 0, bucket_batches = 0, bucket_version = -1;
    std::vector<int> h_bucket_off;  // [n_batches][kDpBuckets+1]
    DpTune tune{{4, 4, 4, 4}, {1, 1, 1, 1}};
    // graph cache
    cudaGraphExec_t graph = nullptr;
    int graph_version = -1, graph_stamp = -1;
    int64_t graph_kernels = 0;
    // timing
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool profiling = false;
    unsigned long long wait_ns = kBarrierTimeoutNs;  // limit of every device-side wait (grb_set_wait_limit)
    unsigned long long* d_phase = nullptr;     // [kPhaseSlots] persistent-kernel phase clocks
    double phase_ms[kPhaseSlots] = {};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    std::vector<int> ev_slot;                  // phase slot of each recorded pair
    size_t ev_used = 0;
    double batching_ms = 0, dag_ms = 0;
    // stage tail (grb_set_stage_tail): buffers grow on demand
    int tail_flags = 0, tail_threshold = 0, tail_nets = 0, tail_valid = 0;
    int* tail_of_sum = nullptr;
    unsigned char* tail_is_of = nullptr;
    int tail_is_of_cap = 0;
    unsigned char* tail_cong = nullptr;
    float *tail_xsum = nullptr, *tail_ysum = nullptr;
};

namespace {

int fail(grb_ctx* c, int code, const std::string& msg) {
    if (c) c->error = msg;
    return code;
}

int cuda_fail(grb_ctx* c, cudaError_t e, const char* what) {
    return fail(c, GRB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GRB_CUDA(ctx, expr)                                             \
    do {                                                                \
        cudaError_t e_ = (expr);                                        \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #expr);      \
    } while (0)

template <class T>
int dalloc(grb_ctx* c, T** p, size_t count, std::vector<void*>& owner) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GRB_ENOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
    }
    owner.push_back(q);
    *p = static_cast<T*>(q);
    return GRB_OK;
}

void free_all(std::vector<void*>& v) {
    for (void* p : v) cudaFree(p);
    v.clear();
}

int check_device_error(grb_ctx* c) {
    int err[2] = {0, 0};
    GRB_CUDA(c, cudaMemcpyAsync(err, c->T.error, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(err + 1, c->T.error_info, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err[0]) {
        GRB_CUDA(c, cudaMemsetAsync(c->T.error, 0, sizeof(int), c->stream));
        switch (err[0]) {
            case kELimit: return fail(c, GRB_ELIMIT, "route storage or colour capacity exceeded (item " + std::to_string(err[1]) + ")");
            case kETimedOut: return fail(c, GRB_ETIMEDOUT, "bounded device wait expired (block " + std::to_string(err[1]) + ")");
            default: return fail(c, GRB_EINVAL, "device reported an invalid state (item " + std::to_string(err[1]) + ")");
        }
    }
    return GRB_OK;
}

Plan make_plan(const grb_ctx* c) {
    Plan P{};
    P.node_off = c->node_off; P.nodes = c->nodes; P.parents = c->parents;
    P.route_off = c->route_off; P.routes = c->routes;
    P.ids = c->ids; P.batch_off = c->batch_off; P.n_batches = c->n_batches;
    P.bucket_ids = c->bucket_ids; P.bucket_off = c->bucket_off;
    return P;
}

// The plan grouped by size bucket, rebuilt when the plan changes (one launch).
int ensure_buckets(grb_ctx* c) {
    if (c->bucket_version == c->plan_version && c->bucket_ids) return GRB_OK;
    if (c->bucket_cap < c->plan_n || c->bucket_batches < c->n_batches || !c->bucket_ids) {
        if (c->bucket_ids) cudaFree(c->bucket_ids);
        if (c->bucket_off) cudaFree(c->bucket_off);
        c->bucket_ids = nullptr; c->bucket_off = nullptr;
        const int cap = std::max(c->plan_n, 1), nb = std::max(c->n_batches, 1);
        if (cudaMalloc(&c->bucket_ids, sizeof(int) * cap) != cudaSuccess ||
            cudaMalloc(&c->bucket_off, sizeof(int) * size_t(nb) * (kDpBuckets + 1)) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GRB_ENOMEM, "bucketed plan");
        }
        c->bucket_cap = cap;
        c->bucket_batches = nb;
    }
    c->h_bucket_off.assign(size_t(c->n_batches) * (kDpBuckets + 1), 0);
    if (c->n_batches) {
        k_plan_buckets<<<c->n_batches, 256, 0, c->stream>>>(make_plan(c), c->bucket_ids, c->bucket_off);
        c->launches += 1;
        GRB_CUDA(c, cudaGetLastError());
        // The per-batch launches are sized from the bucket counts.
        GRB_CUDA(c, cudaMemcpyAsync(c->h_bucket_off.data(), c->bucket_off, sizeof(int) * c->h_bucket_off.size(),
                                    cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    c->bucket_version = c->plan_version;
    return GRB_OK;
}

// The plan with the phase-two routes of the FLT stage.
Plan make_plan2(const grb_ctx* c) {
    Plan P = make_plan(c);
    P.route_off = c->F.route2_off;
    P.routes = c->F.routes2;
    return P;
}

int dp_nmax(const grb_ctx* c) { return std::min(c->max_nodes, 16); }


// Global scratch for nets with more nodes than fit a shared-memory arena of
// `nmax` nodes.
int ensure_gscratch(grb_ctx* c, int slots, int nmax) {
    if (c->max_nodes <= nmax) return GRB_OK;
    const size_t need = size_t(slots) * arena_bytes(c->T.L, c->max_nodes);
    if (need <= c->gscratch_bytes) return GRB_OK;
    if (c->gscratch) cudaFree(c->gscratch);
    c->gscratch = nullptr;
    c->gscratch_bytes = 0;
    if (cudaMalloc(&c->gscratch, need) != cudaSuccess) { cudaGetLastError(); return fail(c, GRB_ENOMEM, "DP scratch allocation failed"); }
    c->gscratch_bytes = need;
    return GRB_OK;
}

// Plain-form profiling: an event pair around each launch group, resolved later.
int prof_begin(grb_ctx* c, int slot, cudaEvent_t* end) {
    *end = nullptr;
    if (!c->profiling) return GRB_OK;
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t a, b;
        GRB_CUDA(c, cudaEventCreate(&a));
        GRB_CUDA(c, cudaEventCreate(&b));
        c->ev_pool.push_back({a, b});
        c->ev_slot.push_back(slot);
    }
    c->ev_slot[c->ev_used] = slot;
    GRB_CUDA(c, cudaEventRecord(c->ev_pool[c->ev_used].first, c->stream));
    *end = c->ev_pool[c->ev_used].second;
    ++c->ev_used;
    return GRB_OK;
}
void prof_end(grb_ctx* c, cudaEvent_t end) {
    if (end) cudaEventRecord(end, c->stream);
}
int prof_collect(grb_ctx* c) {
    if (!c->profiling) return GRB_OK;
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < c->ev_used; ++k) {
        float ms = 0;
        GRB_CUDA(c, cudaEventElapsedTime(&ms, c->ev_pool[k].first, c->ev_pool[k].second));
        c->phase_ms[c->ev_slot[k]] += ms;
    }
    c->ev_used = 0;
    if (c->d_phase) {
        unsigned long long ns[kPhaseSlots];
        GRB_CUDA(c, cudaMemcpy(ns, c->d_phase, sizeof(ns), cudaMemcpyDeviceToHost));
        for (int k = 0; k < kPhaseSlots; ++k) {
            if (k >= kNetTimeSlot + kDpBuckets && k < kNetTimeSlot + 2 * kDpBuckets)
                c->phase_ms[k] = std::max(c->phase_ms[k], ns[k] * 1e-6);  // longest net: a maximum
            else
                c->phase_ms[k] += ns[k] * 1e-6;
        }
        GRB_CUDA(c, cudaMemset(c->d_phase, 0, sizeof(ns)));
    }
    return GRB_OK;
}

int refresh_plain(grb_ctx* c) {
    const Tables T = c->T;
    cudaEvent_t e;
    int rc = prof_begin(c, 4, &e);
    if (rc) return rc;
    k_collect_groups<<<1, 256, 0, c->stream>>>(T);
    k_refresh_cells<<<c->sms * 8, 256, 0, c->stream>>>(T);
    prof_end(c, e);
    if ((rc = prof_begin(c, 7, &e))) return rc;
    k_prefix_pass1<<<c->sms * 8, 256, 8 * prefix_xpose_bytes(), c->stream>>>(T);
    k_prefix_tree<<<c->sms * 2, kRefreshThreads, prefix_smem_bytes(std::max(T.X, T.Y)), c->stream>>>(T);
    k_prefix_pass2<<<c->sms * 8, 256, 8 * prefix_xpose_bytes(), c->stream>>>(T);
    prof_end(c, e);
    c->launches += 5;
    GRB_CUDA(c, cudaGetLastError());
    return GRB_OK;
}

// Batch b in the per-batch DP form: one launch for all its size buckets (or
// only bucket `only` when only >= 0), each bucket with its tuned nets per CTA
// and an arena sized to the bucket.
int launch_buckets(grb_ctx* c, int b, int stamp, int only) {
    const int* bo = c->h_bucket_off.data() + size_t(b) * (kDpBuckets + 1);
    BucketLaunch BL{};
    int blocks = 0, threads = 32;
    size_t smem = 0;
    int gslots = 0;
    for (int bk = 0; bk < kDpBuckets; ++bk) {
        BL.block_off[bk] = blocks;
        const int cnt = (only < 0 || only == bk) ? bo[bk + 1] - bo[bk] : 0;
        BL.per[bk] = c->tune.per_cta[bk];
        BL.nmax[bk] = bk < kDpBuckets - 1 ? std::min(dp_bucket_nodes(bk), std::max(c->max_nodes, 1)) : 0;
        BL.arena[bk] = BL.nmax[bk] ? int(arena_bytes(c->T.L, BL.nmax[bk])) : 0;
        if (bk == 0) BL.arena[0] = int(std::max<size_t>(BL.arena[0], pair_scratch_bytes()));
        if (cnt <= 0) continue;
        // Bucket 0: each warp takes 32 nets (one per lane).
        const int per_block = BL.per[bk] * (bk == 0 ? 32 : 1);
        const int nb = (cnt + per_block - 1) / per_block;
        blocks += nb;
        threads = std::max(threads, 32 * BL.per[bk]);
        smem = std::max(smem, size_t(BL.per[bk]) * BL.arena[bk]);
        if (!BL.nmax[bk]) gslots = nb * BL.per[bk];
    }
    BL.block_off[kDpBuckets] = blocks;
    if (!blocks) return GRB_OK;
    if (gslots) {
        const int rc = ensure_gscratch(c, gslots, dp_nmax(c));
        if (rc) return rc;
    }
    const size_t arena_slot = arena_bytes(c->T.L, std::max(c->max_nodes, 1));
    k_lshape_bucketed<<<blocks, threads, smem, c->stream>>>(c->T, make_plan(c), b, stamp, BL, c->gscratch, arena_slot);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    return GRB_OK;
}

// Per-batch DP launch.
int route_plain(grb_ctx* c, int b, int stamp) {
    if (c->h_batch_off[b + 1] <= c->h_batch_off[b]) return GRB_OK;
    int rc = ensure_buckets(c);
    if (rc) return rc;
    cudaEvent_t e;
    if ((rc = prof_begin(c, 5, &e))) return rc;
    rc = launch_buckets(c, b, stamp, -1);
    prof_end(c, e);
    return rc;
}

int commit_plain(grb_ctx* c, int b, int stamp, int K) {
    const int cnt = c->h_batch_off[b + 1] - c->h_batch_off[b];
    if (cnt <= 0) return GRB_OK;
    const int blocks = std::min((cnt + 3) / 4, 1056);  // demand.cuh:316
    cudaEvent_t e;
    const int prc = prof_begin(c, 6, &e);
    if (prc) return prc;
    k_commit_wires<<<blocks, 128, 0, c->stream>>>(c->T, make_plan(c), b, stamp, K);
    k_commit_vias<<<blocks, 128, 0, c->stream>>>(c->T, make_plan(c), b, stamp, K);
    prof_end(c, e);
    c->launches += 2;
    GRB_CUDA(c, cudaGetLastError());
    return GRB_OK;
}

// The stage tail's device view (buffers sized for the current design).
StageTail make_tail(grb_ctx* c) {
    StageTail t{};
    t.flags = c->tail_flags;
    t.threshold = c->tail_threshold;
    t.n_nets = c->n_nets;
    t.of_sum = c->tail_of_sum;
    t.is_of = c->tail_is_of;
    t.cong = c->tail_cong;
    t.xsum = c->tail_xsum;
    t.ysum = c->tail_ysum;
    return t;
}

// Grow the tail's per-net flags to the uploaded nets (before any launch).
int ensure_tail(grb_ctx* c) {
    if (!(c->tail_flags & kTailRipup) || c->n_nets <= c->tail_is_of_cap) return GRB_OK;
    if (c->tail_is_of) cudaFree(c->tail_is_of);
    c->tail_is_of = nullptr;
    c->tail_is_of_cap = 0;
    if (cudaMalloc(&c->tail_is_of, c->n_nets) != cudaSuccess) { cudaGetLastError(); return fail(c, GRB_ENOMEM, "rip-up flags"); }
    c->tail_is_of_cap = c->n_nets;
    return GRB_OK;
}

// The stage tail as separate launches after the last batch (plain and graph
// forms).
int launch_tail(grb_ctx* c) {
    if (!c->tail_flags) return GRB_OK;
    const StageTail t = make_tail(c);
    const Tables& T = c->T;
    if (t.flags & kTailRipup) {
        int tracks = 0;
        for (int l = 0; l < T.L; ++l) tracks += (((l & 1) ^ T.DIR) ? T.X : T.Y);
        k_mark_overflow<<<(T.cells + 255) / 256, 256, 0, c->stream>>>(T, t.threshold, t.of_sum);
        k_int_prefix<<<(tracks + 127) / 128, 128, 0, c->stream>>>(T, t.of_sum);
        if (c->n_nets)
            k_overflow_nets<<<(c->n_nets + 255) / 256, 256, 0, c->stream>>>(T, make_plan(c), c->n_nets, t.of_sum, t.is_of);
        c->launches += c->n_nets ? 3 : 2;
    }
    if (t.flags & kTailView) {
        k_congestion<<<(T.XY + 255) / 256, 256, 0, c->stream>>>(T, t.cong, t.xsum, t.ysum);
        k_float_line_prefix<<<(T.X + 127) / 128, 128, 0, c->stream>>>(t.ysum, T.X, T.Y, T.Y, 1);  // per x, along y
        k_float_line_prefix<<<(T.Y + 127) / 128, 128, 0, c->stream>>>(t.xsum, T.Y, T.X, 1, T.Y);  // per y, along x
        c->launches += 3;
    }
    GRB_CUDA(c, cudaGetLastError());
    return GRB_OK;
}

int stage_plain(grb_ctx* c, int stamp0) {
    for (int b = 0; b < c->n_batches; ++b) {
        const int stamp = stamp0 + b + 1;
        int rc = refresh_plain(c);
        if (!rc) rc = route_plain(c, b, stamp);
        if (!rc) rc = commit_plain(c, b, stamp, 1);
        if (rc) return rc;
    }
    return GRB_OK;
}

// --- Z-shape stage executors (pipeline_ggr.hpp:119-134) ---------------------
int z_stage_plain(grb_ctx* c, int stamp0) {
    const Plan P = make_plan(c);
    for (int b = 0; b < c->n_batches; ++b) {
        const int cnt = c->h_batch_off[b + 1] - c->h_batch_off[b];
        if (cnt <= 0) continue;
        const int stamp = stamp0 + b + 1;
        int rc;
        if ((rc = refresh_plain(c))) return rc;
        cudaEvent_t e;
        if ((rc = prof_begin(c, 5, &e))) return rc;
        k_zshape_batch<<<cnt, kZThreads, 0, c->stream>>>(c->T, c->Z, P, b);
        prof_end(c, e);
        if ((rc = prof_begin(c, 6, &e))) return rc;
        k_commit_thread_wires<<<(cnt + 255) / 256, 256, 0, c->stream>>>(c->T, P, b, stamp);
        k_commit_thread_vias<<<(cnt + 255) / 256, 256, 0, c->stream>>>(c->T, P, b, stamp);
        prof_end(c, e);
        c->launches += 3;
        GRB_CUDA(c, cudaGetLastError());
    }
    return GRB_OK;
}

int z_stage_graph(grb_ctx* c, int stamp0) {
    const long long key[3] = {c->plan_version, c->z_version, stamp0};
    if (!c->z_graph || !std::equal(key, key + 3, c->z_graph_key)) {
        if (c->z_graph) { cudaGraphExecDestroy(c->z_graph); c->z_graph = nullptr; }
        const int64_t before = c->launches;
        const bool prof = c->profiling;
        c->profiling = false;
        cudaGraph_t g = nullptr;
        GRB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = z_stage_plain(c, stamp0);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->profiling = prof;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&c->z_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(c, ei, "cudaGraphInstantiate");
        c->z_graph_kernels = c->launches - before;
        c->launches = before;
        std::copy(key, key + 3, c->z_graph_key);
    }
    GRB_CUDA(c, cudaGraphLaunch(c->z_graph, c->stream));
    c->launches += c->z_graph_kernels;
    return GRB_OK;
}

int ensure_work(grb_ctx* c);

int z_stage_persistent(grb_ctx* c, int stamp0) {
    if (c->n_batches == 0) return GRB_OK;
    const size_t smem = std::max(prefix_smem_bytes(std::max(c->T.X, c->T.Y)),
                                 size_t(kPersistentThreads / 32) * prefix_xpose_bytes());
    GRB_CUDA(c, cudaFuncSetAttribute(k_zshape_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    GRB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zshape_persistent, kPersistentThreads, smem));
    if (per_sm < 1) return fail(c, GRB_EINVAL, "persistent Z-shape kernel does not fit on an SM");
    int rc = ensure_work(c);
    if (rc) return rc;
    GRB_CUDA(c, cudaMemsetAsync(c->sync, 0, 2 * sizeof(unsigned), c->stream));
    Tables T = c->T;
    ZTrees Z = c->Z;
    Plan P = make_plan(c);
    GridSync S{c->sync, c->sync + 1, c->wait_ns, c->profiling ? c->d_phase : nullptr};
    void* args[] = {&T, &Z, &P, &S, &stamp0, &c->work};
    GRB_CUDA(c, cudaLaunchCooperativeKernel((void*)k_zshape_persistent, dim3(per_sm * c->sms), dim3(kPersistentThreads),
                                            args, smem, c->stream));
    c->launches += 1;
    return GRB_OK;
}

// --- soft-min executors ------------------------------------------------------
int soft_workspace(grb_ctx* c) {
    const size_t cells = c->T.cells;
    // Range tables and adjoints of every node: 2 * nodes * L * L values.
    const size_t slot = 2 * size_t(std::max(c->topo_sizes[0], 1ll)) * c->T.L * c->T.L * sizeof(double);
    if (c->soft_cells && c->soft_slot_bytes >= slot) return GRB_OK;
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    free_all(c->used_bufs);
    free_all(c->soft_bufs);
    int rc = 0;
    rc |= dalloc(c, &c->soft_cells, 6 * cells * sizeof(double), c->soft_bufs);
    rc |= dalloc(c, &c->soft_slot, slot, c->soft_bufs);
    rc |= dalloc(c, &c->soft_scalar, 2, c->soft_bufs);
    if (rc) { free_all(c->soft_bufs); c->soft_cells = nullptr; return GRB_ENOMEM; }
    c->soft_slot_bytes = slot;
    return GRB_OK;
}

template <class T>
Soft<T> soft_view(grb_ctx* c, double tau, const void* cap, const void* uw, double uv, T* net_cost) {
    const size_t cells = c->T.cells;
    T* a = reinterpret_cast<T*>(c->soft_cells);
    Soft<T> S{};
    S.cap = static_cast<const T*>(cap);
    S.uw = static_cast<const T*>(uw);
    S.uv = static_cast<T>(uv);
    S.tau = static_cast<T>(tau);
    S.wc = a; S.vc = a + cells; S.P = a + 2 * cells; S.dP = a + 3 * cells; S.dvc = a + 4 * cells;
    S.slot = reinterpret_cast<T*>(c->soft_slot);
    S.net_cost = net_cost;
    return S;
}

template <class T>
int soft_forward(grb_ctx* c, double tau, const void* cap, const void* uw, double uv, T* net_cost, double* total) {
    const Tables& Tb = c->T;
    const int n = c->n_nets;
    Soft<T> S = soft_view<T>(c, tau, cap, uw, uv, net_cost);
    const int M = std::max(Tb.X, Tb.Y);
    k_soft_tables<T><<<(Tb.cells + 255) / 256, 256, 0, c->stream>>>(Tb, S);
    k_soft_prefix<T><<<(Tb.L * M + 127) / 128, 128, 0, c->stream>>>(Tb, S);
    k_soft_forward<T><<<std::max(1, (n + kSoftThreads - 1) / kSoftThreads), kSoftThreads, 0, c->stream>>>(
        Tb, S, make_plan(c), n);
    k_soft_sum<T><<<1, 1024, 0, c->stream>>>(net_cost, n, c->soft_scalar);
    c->launches += 4;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaMemcpyAsync(total, c->soft_scalar, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

template <class T>
int soft_backward(grb_ctx* c, double tau, const void* cap, const void* uw, double uv, double g, T* dcap, T* duw,
                  double* duv) {
    const Tables& Tb = c->T;
    const int n = c->n_nets;
    const size_t cells = Tb.cells;
    Soft<T> S = soft_view<T>(c, tau, cap, uw, uv, nullptr);
    T* dwc = reinterpret_cast<T*>(c->soft_cells) + 5 * cells;
    const int M = std::max(Tb.X, Tb.Y);
    k_soft_tables<T><<<(Tb.cells + 255) / 256, 256, 0, c->stream>>>(Tb, S);
    k_soft_prefix<T><<<(Tb.L * M + 127) / 128, 128, 0, c->stream>>>(Tb, S);
    GRB_CUDA(c, cudaMemsetAsync(S.dP, 0, sizeof(T) * cells, c->stream));
    GRB_CUDA(c, cudaMemsetAsync(S.dvc, 0, sizeof(T) * cells, c->stream));
    k_soft_backward<T><<<std::max(1, (n + kSoftThreads - 1) / kSoftThreads), kSoftThreads, 0, c->stream>>>(
        Tb, S, make_plan(c), n, static_cast<T>(g));
    k_soft_suffix<T><<<(Tb.L * M + 127) / 128, 128, 0, c->stream>>>(Tb, S, dwc);
    k_soft_chain<T><<<(Tb.cells + 255) / 256, 256, 0, c->stream>>>(Tb, S, dwc, dcap, duw);
    k_soft_sum<T><<<1, 1024, 0, c->stream>>>(S.dvc, int(cells), c->soft_scalar + 1);
    c->launches += 6;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaMemcpyAsync(duv, c->soft_scalar + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

// --- FLT stage executors ---------------------------------------------------
int flt_stamps(const grb_ctx* c, int remove) { return c->n_batches * (remove ? 2 : 1); }

int flt_stage_plain(grb_ctx* c, int stamp0, int remove) {
    const Plan P1 = make_plan(c), P2 = make_plan2(c);
    for (int b = 0; b < c->n_batches; ++b) {
        const int cnt = c->h_batch_off[b + 1] - c->h_batch_off[b];
        if (cnt <= 0) continue;
        const int stamp = stamp0 + (remove ? 2 * b + 2 : b + 1);
        const int cblocks = std::min((cnt + 3) / 4, 1056);  // demand.cuh:316
        int rc;
        cudaEvent_t e;
        if (remove) {  // flt.cuh:143-150
            if ((rc = prof_begin(c, 6, &e))) return rc;
            k_commit_wires<<<cblocks, 128, 0, c->stream>>>(c->T, P1, b, stamp - 1, -1);
            k_commit_vias<<<cblocks, 128, 0, c->stream>>>(c->T, P1, b, stamp - 1, -1);
            prof_end(c, e);
            c->launches += 2;
        }
        if ((rc = refresh_plain(c))) return rc;
        if ((rc = prof_begin(c, 5, &e))) return rc;
        k_flt_edges<<<c->sms * 8, 256, 0, c->stream>>>(c->T, c->F, P2, b);
        c->launches += 1;
        const int nw = c->h_flt_nwide[b];
        k_flt_batch<<<nw + (cnt - nw + kFltThreads / 32 - 1) / (kFltThreads / 32), kFltThreads, 0, c->stream>>>(
            c->T, c->F, P2, b, stamp, nw);
        prof_end(c, e);
        if ((rc = prof_begin(c, 6, &e))) return rc;
        k_commit_vias<<<cblocks, 128, 0, c->stream>>>(c->T, P2, b, stamp, 1);
        prof_end(c, e);
        c->launches += 2;
        GRB_CUDA(c, cudaGetLastError());
    }
    return GRB_OK;
}

int flt_stage_graph(grb_ctx* c, int stamp0, int remove) {
    const long long key[5] = {c->plan_version, c->flt_version, stamp0, remove, c->flt_block_width};
    if (!c->flt_graph || !std::equal(key, key + 5, c->flt_graph_key)) {
        if (c->flt_graph) { cudaGraphExecDestroy(c->flt_graph); c->flt_graph = nullptr; }
        const int64_t before = c->launches;
        const bool prof = c->profiling;
        c->profiling = false;
        cudaGraph_t g = nullptr;
        GRB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = flt_stage_plain(c, stamp0, remove);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->profiling = prof;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&c->flt_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(c, ei, "cudaGraphInstantiate");
        c->flt_graph_kernels = c->launches - before;
        c->launches = before;
        std::copy(key, key + 5, c->flt_graph_key);
    }
    GRB_CUDA(c, cudaGraphLaunch(c->flt_graph, c->stream));
    c->launches += c->flt_graph_kernels;
    return GRB_OK;
}

int ensure_work(grb_ctx* c) {
    if (c->work_cap < c->n_batches) {
        if (c->work) cudaFree(c->work);
        c->work = nullptr;
        if (cudaMalloc(&c->work, sizeof(int) * c->n_batches) != cudaSuccess) { cudaGetLastError(); return fail(c, GRB_ENOMEM, "work counters"); }
        c->work_cap = c->n_batches;
    }
    GRB_CUDA(c, cudaMemsetAsync(c->work, 0, sizeof(int) * std::max(c->n_batches, 1), c->stream));
    return GRB_OK;
}

int flt_stage_persistent(grb_ctx* c, int stamp0, int remove) {
    if (c->n_batches == 0) return GRB_OK;
    const size_t smem = std::max(prefix_smem_bytes(std::max(c->T.X, c->T.Y)),
                                 size_t(kPersistentThreads / 32) * prefix_xpose_bytes());
    GRB_CUDA(c, cudaFuncSetAttribute(k_flt_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    GRB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flt_persistent, kPersistentThreads, smem));
    if (per_sm < 1) return fail(c, GRB_EINVAL, "persistent FLT kernel does not fit on an SM");
    int rc = ensure_work(c);
    if (rc) return rc;
    GRB_CUDA(c, cudaMemsetAsync(c->sync, 0, 2 * sizeof(unsigned), c->stream));
    Tables T = c->T;
    Flt F = c->F;
    Plan P1 = make_plan(c), P2 = make_plan2(c);
    GridSync S{c->sync, c->sync + 1, c->wait_ns, c->profiling ? c->d_phase : nullptr};
    void* args[] = {&T, &F, &P1, &P2, &S, &stamp0, &remove, &c->work};
    GRB_CUDA(c, cudaLaunchCooperativeKernel((void*)k_flt_persistent, dim3(per_sm * c->sms), dim3(kPersistentThreads),
                                            args, smem, c->stream));
    c->launches += 1;
    return GRB_OK;
}

int stage_graph(grb_ctx* c, int stamp0) {
    if (!c->graph || c->graph_version != c->plan_version || c->graph_stamp != stamp0) {
        if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
        // Scratch must exist before capture (no allocation while capturing).
        int maxcnt = 0;
        for (int b = 0; b < c->n_batches; ++b) maxcnt = std::max(maxcnt, c->h_batch_off[b + 1] - c->h_batch_off[b]);
        int rc = ensure_gscratch(c, maxcnt + 8, dp_nmax(c));
        if (!rc) rc = ensure_buckets(c);
        if (rc) return rc;
        const int64_t before = c->launches;
        const bool prof = c->profiling;
        c->profiling = false;
        cudaGraph_t g = nullptr;
        GRB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        rc = stage_plain(c, stamp0);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->profiling = prof;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(c, ei, "cudaGraphInstantiate");
        c->graph_kernels = c->launches - before;
        c->launches = before;
        c->graph_version = c->plan_version;
        c->graph_stamp = stamp0;
    }
    GRB_CUDA(c, cudaGraphLaunch(c->graph, c->stream));
    c->launches += c->graph_kernels;
    return GRB_OK;
}

int stage_persistent(grb_ctx* c, int stamp0) {
    if (c->n_batches == 0) return GRB_OK;
    const int nmax = dp_nmax(c);
    // A warp's arena also holds the lane-per-net scratch of the smallest nets.
    const size_t ab = std::max(arena_bytes(c->T.L, nmax), (pair_scratch_bytes() + 15) & ~size_t(15));
    const int wpb = kPersistentThreads / 32;
    const size_t prefix_smem = prefix_smem_bytes(std::max(c->T.X, c->T.Y));  // prefix_tree
    const size_t smem = std::max(std::max(ab * wpb, prefix_smem), size_t(wpb) * prefix_xpose_bytes());
    GRB_CUDA(c, cudaFuncSetAttribute(k_lshape_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    GRB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lshape_persistent, kPersistentThreads, smem));
    if (per_sm < 1) return fail(c, GRB_EINVAL, "persistent kernel does not fit on an SM");
    const int blocks = per_sm * c->sms;
    const size_t slot = arena_bytes(c->T.L, std::max(c->max_nodes, 1));
    int rc = ensure_gscratch(c, blocks * wpb, nmax);
    if (rc) return rc;
    if ((rc = ensure_buckets(c))) return rc;
    const int counters = c->n_batches * kDpBuckets;
    if (c->work_cap < counters) {
        if (c->work) cudaFree(c->work);
        c->work = nullptr;
        if (cudaMalloc(&c->work, sizeof(int) * counters) != cudaSuccess) { cudaGetLastError(); return fail(c, GRB_ENOMEM, "work counters"); }
        c->work_cap = counters;
    }
    GRB_CUDA(c, cudaMemsetAsync(c->work, 0, sizeof(int) * counters, c->stream));
    GRB_CUDA(c, cudaMemsetAsync(c->sync, 0, 2 * sizeof(unsigned), c->stream));
    Tables T = c->T;
    Plan P = make_plan(c);
    GridSync S{c->sync, c->sync + 1, c->wait_ns, c->profiling ? c->d_phase : nullptr};
    char* gs = c->gscratch;
    DpTune tune = c->tune;
    if ((rc = ensure_tail(c))) return rc;
    StageTail tail = make_tail(c);
    void* args[] = {&T, &P, &S, &stamp0, (void*)&nmax, (void*)&ab, &gs, (void*)&slot, &c->work, &tune, &tail};
    GRB_CUDA(c, cudaLaunchCooperativeKernel((void*)k_lshape_persistent, dim3(blocks), dim3(kPersistentThreads), args, smem, c->stream));
    c->launches += 1;
    return GRB_OK;
}

int ensure_plan_capacity(grb_ctx* c, int n, int nb) {
    if (c->ids && n <= c->plan_cap && nb + 1 <= c->plan_cap + 1) {
        return GRB_OK;
    }
    if (c->ids) cudaFree(c->ids);
    if (c->batch_off) cudaFree(c->batch_off);
    c->ids = nullptr; c->batch_off = nullptr;
    const int cap = std::max(n, 1);
    if (cudaMalloc(&c->ids, sizeof(int) * cap) != cudaSuccess ||
        cudaMalloc(&c->batch_off, sizeof(int) * (size_t(cap) + 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GRB_ENOMEM, "plan allocation failed");
    }
    c->plan_cap = cap;
    return GRB_OK;
}

// Runs the batching of B (chunks of CH nets) in the requested form.
template <int CH>
static int launch_batching(grb_ctx* c, BatchState& B, int mode, size_t smem) {
    const int n = B.n;
    int rc = GRB_OK;
    int per_sm = 0;
    if (mode == GRB_MODE_PERSISTENT)
        GRB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent<CH>, kPersistThreads, smem));
    if (mode == GRB_MODE_PERSISTENT && per_sm * c->sms >= 2) {
        GRB_CUDA(c, cudaMemsetAsync(c->sync, 0, 2 * sizeof(unsigned), c->stream));
        GridSync S{c->sync, c->sync + 1, c->wait_ns, c->profiling ? c->d_phase : nullptr, 0};
        Tables T = c->T;
        void* args[] = {&B, &S, &T};
        GRB_CUDA(c, cudaLaunchCooperativeKernel((void*)k_batch_persistent<CH>, dim3(per_sm * c->sms), dim3(kPersistThreads),
                                                args, smem, c->stream));
        c->launches += 1;
        return GRB_OK;
    }
    const int grid = c->sms * 4;
    if (n) k_batch_point_bits<CH><<<grid, 256, 0, c->stream>>>(B, 0);
    c->launches += n ? 1 : 0;
    for (int s = 0; s < n; s += CH) {
        cudaEvent_t e;
        if ((rc = prof_begin(c, 0, &e))) return rc;
        k_batch_raster<CH><<<grid, 256, 0, c->stream>>>(B, s);
        prof_end(c, e);
        if ((rc = prof_begin(c, 1, &e))) return rc;
        k_batch_gather<CH><<<grid, 256, 0, c->stream>>>(B, s);
        prof_end(c, e);
        if ((rc = prof_begin(c, 2, &e))) return rc;
        k_batch_solve<CH><<<1, CH, smem, c->stream>>>(B, s);
        prof_end(c, e);
        if ((rc = prof_begin(c, 3, &e))) return rc;
        k_batch_publish<CH><<<grid, 256, 0, c->stream>>>(B, s);
        prof_end(c, e);
        c->launches += 4;
    }
    GRB_CUDA(c, cudaGetLastError());
    return GRB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int grb_init_device(int32_t device) {
    if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
        cudaGetLastError();
        return GRB_ECUDA;
    }
    // Loading a kernel's code is deferred to its first use; these are the
    // kernels every stage starts with.
    const void* kernels[] = {(const void*)k_batch_persistent<kChunkMax>, (const void*)k_lshape_persistent,
                             (const void*)k_flt_persistent, (const void*)k_zshape_persistent,
                             (const void*)k_refresh_cells, (const void*)k_prefix_pass1, (const void*)k_prefix_pass2,
                             (const void*)k_lshape_bucketed, (const void*)k_topo_fill, (const void*)k_out_write};
    for (const void* k : kernels) {
        cudaFuncAttributes a{};
        if (cudaFuncGetAttributes(&a, k) != cudaSuccess) {
            cudaGetLastError();
            return GRB_ECUDA;
        }
    }
    return GRB_OK;
}

int grb_create(const grb_grid* g, int32_t device, grb_ctx** out) {
    if (!out) return GRB_EINVAL;
    *out = nullptr;
    if (!g || g->L < 1 || g->L > kMaxLayers || g->X < 2 || g->Y < 2 || !g->capacity ||
        !g->unit_length_short_costs || !g->x_edge_len || !g->y_edge_len)
        return GRB_EINVAL;
    if (size_t(g->L) * g->X * g->Y >= (size_t(1) << 31)) return GRB_EINVAL;
    if (std::max(g->X, g->Y) > 8192) return GRB_EINVAL;  // prefix tree depth (kChunkPos << 8)
    auto c = std::make_unique<grb_ctx>();
    c->device = device;
    GRB_CUDA(c.get(), cudaSetDevice(device));
    GRB_CUDA(c.get(), cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    GRB_CUDA(c.get(), cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    GRB_CUDA(c.get(), cudaEventCreate(&c->ev0));
    GRB_CUDA(c.get(), cudaEventCreate(&c->ev1));
    Tables& T = c->T;
    T.L = g->L; T.X = g->X; T.Y = g->Y; T.DIR = g->DIR & 1; T.XY = g->X * g->Y;
    T.cells = T.L * T.XY;
    T.unit_wire = g->unit_length_wire_cost; T.unit_via = g->unit_via_cost;
    T.of_scale = g->of_cost_scale;
    const size_t cells = T.cells;
    T.words = int((cells + 31) / 32);
    int ng = 0;
    for (int l = 0; l < T.L; ++l) {
        T.group_base[l] = ng;
        const int tracks = (((l & 1) ^ T.DIR) ? T.X : T.Y);
        ng += (tracks + kTrackGroup - 1) / kTrackGroup;
    }
    T.group_base[T.L] = ng;
    for (int l = T.L + 1; l <= kMaxLayers; ++l) T.group_base[l] = ng;
    T.n_groups = ng;
    grb_ctx* cp = c.get();
    double* sc; int* xl; int* yl; float* cap;
    int rc = 0;
    rc |= dalloc(cp, &sc, T.L, cp->owned);
    rc |= dalloc(cp, &xl, T.X - 1, cp->owned);
    rc |= dalloc(cp, &yl, T.Y - 1, cp->owned);
    rc |= dalloc(cp, &cap, cells, cp->owned);
    rc |= dalloc(cp, &T.demand, cells, cp->owned);
    rc |= dalloc(cp, &T.ts, cells, cp->owned);
    rc |= dalloc(cp, &T.wcost, cells, cp->owned);
    rc |= dalloc(cp, &T.vcost, cells, cp->owned);
    rc |= dalloc(cp, &T.presum, cells, cp->owned);
    rc |= dalloc(cp, &T.dirty_wire, T.words, cp->owned);
    rc |= dalloc(cp, &T.dirty_via, T.words, cp->owned);
    rc |= dalloc(cp, &T.group_first, ng, cp->owned);
    rc |= dalloc(cp, &T.first_list, ng, cp->owned);
    rc |= dalloc(cp, &T.group_list, ng, cp->owned);
    rc |= dalloc(cp, &T.group_count, 1, cp->owned);
    T.tree_chunks = prefix_chunks(std::max(T.X, T.Y));
    T.tree_stride = prefix_tree_entries(std::max(T.X, T.Y));
    rc |= dalloc(cp, &T.ptree, size_t(ng) * T.tree_stride * 32, cp->owned);

    rc |= dalloc(cp, &T.wirelength, 1, cp->owned);
    rc |= dalloc(cp, &T.vias, 1, cp->owned);
    rc |= dalloc(cp, &T.error, 2, cp->owned);
    rc |= dalloc(cp, &c->sync, 2, cp->owned);
    if (rc) { free_all(cp->owned); return GRB_ENOMEM; }
    T.error_info = T.error + 1;
    T.short_costs = sc; T.xlen = xl; T.ylen = yl; T.capacity = cap;
    GRB_CUDA(cp, cudaMemcpy(sc, g->unit_length_short_costs, sizeof(double) * T.L, cudaMemcpyHostToDevice));
    GRB_CUDA(cp, cudaMemcpy(xl, g->x_edge_len, sizeof(int) * (T.X - 1), cudaMemcpyHostToDevice));
    GRB_CUDA(cp, cudaMemcpy(yl, g->y_edge_len, sizeof(int) * (T.Y - 1), cudaMemcpyHostToDevice));
    GRB_CUDA(cp, cudaMemcpy(cap, g->capacity, sizeof(float) * cells, cudaMemcpyHostToDevice));
    GRB_CUDA(cp, cudaMemset(T.error, 0, 2 * sizeof(int)));
    {
        // Distinct capacity values (at most kNoCapRow of them get table rows;
        // with more, every cost is computed) and each cell's row.
        std::vector<unsigned char> cid(cells);
        std::vector<float> caps;
        std::unordered_map<uint32_t, int> row;
        uint32_t last = 0;
        int last_row = -1;
        for (size_t i = 0; i < cells; ++i) {
            uint32_t bits;
            std::memcpy(&bits, g->capacity + i, 4);
            if (last_row < 0 || bits != last) {
                auto it = row.find(bits);
                if (it == row.end()) {
                    if (int(caps.size()) >= kNoCapRow) { caps.clear(); break; }
                    it = row.emplace(bits, int(caps.size())).first;
                    caps.push_back(g->capacity[i]);
                }
                last = bits;
                last_row = it->second;
            }
            cid[i] = static_cast<unsigned char>(last_row);
        }
        if (caps.empty()) std::fill(cid.begin(), cid.end(), static_cast<unsigned char>(kNoCapRow));
        unsigned char* d_cid = nullptr;
        double2* d_table = nullptr;
        float* d_caps = nullptr;
        const int rows = std::max<int>(int(caps.size()), 1);
        T.of_dmax = caps.empty() ? 0 : kOfDmax;
        T.of_rows = rows;
        T.of_stride = kOfDmax;
        if (dalloc(cp, &d_cid, cells, cp->owned) ||
            dalloc(cp, &d_table, size_t(T.L) * rows * T.of_stride, cp->owned) || dalloc(cp, &d_caps, rows, cp->owned)) {
            free_all(cp->owned);
            return GRB_ENOMEM;
        }
        T.cap_id = d_cid;
        T.of_table = d_table;
        GRB_CUDA(cp, cudaMemcpy(d_cid, cid.data(), cells, cudaMemcpyHostToDevice));
        if (!caps.empty()) {
            GRB_CUDA(cp, cudaMemcpy(d_caps, caps.data(), sizeof(float) * caps.size(), cudaMemcpyHostToDevice));
            const int n = T.L * rows * T.of_stride;
            k_build_of_table<<<(n + 255) / 256, 256>>>(T, d_caps);
            GRB_CUDA(cp, cudaGetLastError());
            GRB_CUDA(cp, cudaDeviceSynchronize());
        }
    }
    GRB_CUDA(cp, cudaFuncSetAttribute(k_batch_solve<kChunkMax>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSolveSmemLimit)));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_batch_solve<kChunkMax / 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSolveSmemLimit)));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_batch_persistent<kChunkMax>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSolveSmemLimit)));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_batch_persistent<kChunkMax / 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSolveSmemLimit)));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_lshape_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_lshape_bucketed, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_prefix_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(8 * prefix_xpose_bytes())));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_prefix_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize, int(8 * prefix_xpose_bytes())));
    GRB_CUDA(cp, cudaFuncSetAttribute(k_prefix_tree, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(prefix_smem_bytes(std::max(T.X, T.Y)))));
    const int r = grb_reset(cp);
    if (r) { const int code = r; free_all(cp->owned); return code; }
    *out = c.release();
    return GRB_OK;
}

void grb_destroy(grb_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* p : {(void*)c->tail_of_sum, (void*)c->tail_is_of, (void*)c->tail_cong, (void*)c->tail_xsum,
                    (void*)c->tail_ysum})
        if (p) cudaFree(p);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->flt_graph) cudaGraphExecDestroy(c->flt_graph);
    if (c->z_graph) cudaGraphExecDestroy(c->z_graph);
    free_all(c->soft_bufs);
    free_all(c->z_bufs);
    free_all(c->box_bufs);
    free_all(c->net_bufs);
    free_all(c->geom_bufs);
    free_all(c->flt_bufs);
    free_all(c->topo_bufs);
    if (c->out_stream) cudaStreamSynchronize(c->out_stream);
    free_all(c->out_bufs);
    if (c->out_text) cudaFree(c->out_text);
    for (char* h : c->out_host)
        if (h) cudaFreeHost(h);
    for (cudaEvent_t e : {c->out_ready, c->out_chunk_ev[0], c->out_chunk_ev[1]})
        if (e) cudaEventDestroy(e);
    if (c->out_stream) cudaStreamDestroy(c->out_stream);
    if (c->flt_eprefix) cudaFree(c->flt_eprefix);
    if (c->flt_emap) cudaFree(c->flt_emap);
    if (c->flt_border) cudaFree(c->flt_border);
    if (c->flt_nwide) cudaFree(c->flt_nwide);
    if (c->ckpt_demand) cudaFree(c->ckpt_demand);
    if (c->score_partials) cudaFree(c->score_partials);
    free_all(c->owned);
    for (void* p : {(void*)c->check, (void*)c->bucket_ids, (void*)c->bucket_off, (void*)c->ids, (void*)c->batch_off, (void*)c->gscratch, (void*)c->work, (void*)c->cellmask,
                    (void*)c->lmask[0], (void*)c->lmask[1], (void*)c->lmask[2], (void*)c->lmask[3], (void*)c->lmask[4],
                    (void*)c->ptchunk, (void*)c->fmask, (void*)c->pred, (void*)c->prevp,
                    (void*)c->bsolved, (void*)c->fullmask, (void*)c->bcount, (void*)c->ncolors, (void*)c->batch_of, (void*)c->brank,
                    (void*)c->order, (void*)c->rank_tiles, (void*)c->mark_off, (void*)c->pt_off, (void*)c->scan_sums, (void*)c->mark_cell,
                    (void*)c->pt_cell, (void*)c->mark_jj, (void*)c->pt_jj})
        if (p) cudaFree(p);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* grb_last_error(const grb_ctx* c) { return c ? c->error.c_str() : "null context"; }

void* grb_stream(grb_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int grb_reset(grb_ctx* c) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    Tables& T = c->T;
    const size_t cells = T.cells;
    GRB_CUDA(c, cudaMemsetAsync(T.demand, 0, sizeof(int) * cells, c->stream));
    GRB_CUDA(c, cudaMemsetAsync(T.ts, 0, sizeof(int) * cells, c->stream));
    GRB_CUDA(c, cudaMemsetAsync(T.wirelength, 0, sizeof(double), c->stream));
    GRB_CUDA(c, cudaMemsetAsync(T.vias, 0, sizeof(unsigned long long), c->stream));
    if (c->routes) GRB_CUDA(c, cudaMemsetAsync(c->routes, 0, sizeof(int) * std::max<long long>(c->route_words, 1), c->stream));
    const int n = std::max(T.words, T.n_groups);
    k_mark_all_dirty<<<(n + 255) / 256, 256, 0, c->stream>>>(T);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    c->stamp = 0;
    return GRB_OK;
}

// Device buffers of the net store, reused while every array still fits
// (need: nets, nodes, route words, points, h-segments, v-segments).
static int net_buffers(grb_ctx* c, const long long need[6]) {
    bool fits = !c->net_bufs.empty() && c->geom_bufs.empty();
    for (int k = 0; k < 6 && fits; ++k) fits = need[k] <= c->net_cap[k];
    if (fits) return GRB_OK;
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    free_all(c->net_bufs);
    free_all(c->geom_bufs);
    free_all(c->flt_bufs);
    c->flt_n = -1;
    const long long n = need[0], nn = need[1], rw = need[2], np = need[3], nh = need[4], nv = need[5];
    int rc = 0;
    rc |= dalloc(c, &c->node_off, n + 1, c->net_bufs);
    rc |= dalloc(c, &c->nodes, nn, c->net_bufs);
    rc |= dalloc(c, &c->parents, nn, c->net_bufs);
    rc |= dalloc(c, &c->route_off, n + 1, c->net_bufs);
    rc |= dalloc(c, &c->routes, rw, c->net_bufs);
    rc |= dalloc(c, &c->point_off, n + 1, c->net_bufs);
    rc |= dalloc(c, &c->points, np, c->net_bufs);
    rc |= dalloc(c, &c->hseg_off, n + 1, c->net_bufs);
    rc |= dalloc(c, &c->hsegs, 2 * size_t(nh), c->net_bufs);
    rc |= dalloc(c, &c->vseg_off, n + 1, c->net_bufs);
    rc |= dalloc(c, &c->vsegs, 2 * size_t(nv), c->net_bufs);
    if (rc) { free_all(c->net_bufs); return fail(c, GRB_ENOMEM, "net buffers"); }
    for (int k = 0; k < 6; ++k) c->net_cap[k] = need[k];
    return GRB_OK;
}

// Device-side check of the net store just written (every index a stage kernel
// will dereference); the net count becomes the context's on success.
static int validate_net_store(grb_ctx* c, int n, int nn, long long rw, int np, int nh, int nv) {
    int status[3] = {0, 0, 0};
    if (!c->check) {
        if (cudaMalloc(&c->check, 3 * sizeof(int)) != cudaSuccess) { cudaGetLastError(); return fail(c, GRB_ENOMEM, "validation status"); }
    }
    GRB_CUDA(c, cudaMemsetAsync(c->check, 0, 3 * sizeof(int), c->stream));
    NetCheck C{c->node_off, c->nodes, c->parents, c->route_off, c->point_off, c->points, c->hseg_off, c->hsegs,
               c->vseg_off, c->vsegs, n, nn, np, nh, nv, c->T.XY, c->T.L, rw, c->check};
    k_validate_nets<<<c->sms * 4, 256, 0, c->stream>>>(C);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaMemcpyAsync(status, c->check, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->flt_n = -1;  // FLT DAGs and Z-shape trees refer to the previous nets
    c->z_n = -1;
    if (status[0]) {
        static const char* what[] = {"", "offsets must be non-decreasing and within the arrays", "tree node outside the grid",
                                     "parents must precede children", "batching geometry outside the grid"};
        c->n_nets = 0;  // no net id is accepted until a valid upload
        c->topo_sizes[0] = -1;
        return fail(c, GRB_EINVAL, std::string(what[status[0]]) + " (item " + std::to_string(status[1]) + ")");
    }
    c->n_nets = n;
    c->max_nodes = status[2];
    c->route_words = rw;
    c->topo_sizes[0] = nn;
    c->topo_sizes[1] = np;
    c->topo_sizes[2] = nh;
    c->topo_sizes[3] = nv;
    return GRB_OK;
}

int grb_upload_nets(grb_ctx* c, const grb_nets* nets) {
    if (!c || !nets || nets->n < 0 || !nets->node_off || !nets->route_off) return c ? fail(c, GRB_EINVAL, "bad nets") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = nets->n;
    // Only the totals are read on the host (they size the buffers); every
    // element is checked on the device after the upload.
    if (nets->node_off[0] != 0 || nets->route_off[0] != 0 || (nets->point_off && nets->point_off[0] != 0) ||
        (nets->hseg_off && nets->hseg_off[0] != 0) || (nets->vseg_off && nets->vseg_off[0] != 0))
        return fail(c, GRB_EINVAL, "offsets must start at 0");
    const int nn = nets->node_off[n];
    const long long rw = nets->route_off[n];
    const int np = nets->point_off ? nets->point_off[n] : 0;
    const int nh = nets->hseg_off ? nets->hseg_off[n] : 0;
    const int nv = nets->vseg_off ? nets->vseg_off[n] : 0;
    if (nn < 0 || rw < 0 || np < 0 || nh < 0 || nv < 0) return fail(c, GRB_EINVAL, "negative totals");
    if ((nn && (!nets->nodes || !nets->parents)) || (np && !nets->points) || (nh && !nets->hsegs) || (nv && !nets->vsegs))
        return fail(c, GRB_EINVAL, "net arrays missing");
    const long long need[6] = {n, nn, rw, np, nh, nv};
    if (int rc = net_buffers(c, need)) return rc;
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return src && bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, h2d(c->node_off, nets->node_off, sizeof(int) * (n + 1)));
    GRB_CUDA(c, h2d(c->nodes, nets->nodes, sizeof(int) * nn));
    GRB_CUDA(c, h2d(c->parents, nets->parents, sizeof(int) * nn));
    GRB_CUDA(c, h2d(c->route_off, nets->route_off, sizeof(long long) * (n + 1)));
    GRB_CUDA(c, cudaMemsetAsync(c->routes, 0, sizeof(int) * std::max<long long>(rw, 1), c->stream));
    if (nets->point_off) GRB_CUDA(c, h2d(c->point_off, nets->point_off, sizeof(int) * (n + 1)));
    else GRB_CUDA(c, cudaMemsetAsync(c->point_off, 0, sizeof(int) * (n + 1), c->stream));
    GRB_CUDA(c, h2d(c->points, nets->points, sizeof(int) * np));
    if (nets->hseg_off) GRB_CUDA(c, h2d(c->hseg_off, nets->hseg_off, sizeof(int) * (n + 1)));
    else GRB_CUDA(c, cudaMemsetAsync(c->hseg_off, 0, sizeof(int) * (n + 1), c->stream));
    GRB_CUDA(c, h2d(c->hsegs, nets->hsegs, sizeof(int) * 2 * nh));
    if (nets->vseg_off) GRB_CUDA(c, h2d(c->vseg_off, nets->vseg_off, sizeof(int) * (n + 1)));
    else GRB_CUDA(c, cudaMemsetAsync(c->vseg_off, 0, sizeof(int) * (n + 1), c->stream));
    GRB_CUDA(c, h2d(c->vsegs, nets->vsegs, sizeof(int) * 2 * nv));
    // Host buffers may be pageable and short-lived: the validation's
    // synchronisation completes the copies before return.
    return validate_net_store(c, n, nn, rw, np, nh, nv);
}

int grb_build_topology(grb_ctx* c, const grb_trees* t) {
    if (!c || !t || t->n < 0 || !t->node_off || !t->route_off || !t->adj_off)
        return c ? fail(c, GRB_EINVAL, "bad trees") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = t->n;
    if (t->node_off[0] != 0 || t->route_off[0] != 0 || t->adj_off[0] != 0)
        return fail(c, GRB_EINVAL, "offsets must start at 0");
    const long long nn = t->node_off[n], rw = t->route_off[n];
    if (nn < 0 || nn > (1ll << 30) || rw < 0) return fail(c, GRB_EINVAL, "bad totals");
    const long long na = t->adj_off[nn];
    if (na < 0 || (nn && !t->pos) || (na && !t->adj)) return fail(c, GRB_EINVAL, "tree arrays missing");
    // Uploaded trees, per-net counts and the DFS stack (freed after the build).
    free_all(c->topo_bufs);
    int *d_node_off = nullptr, *d_pos = nullptr, *d_adj_off = nullptr, *d_adj = nullptr, *d_stack = nullptr,
        *d_status = nullptr;
    long long *d_cnt = nullptr, *d_sums = nullptr;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    int rc = 0;
    rc |= dalloc(c, &d_node_off, n + 1, c->topo_bufs);
    rc |= dalloc(c, &d_pos, std::max(nn, 1ll), c->topo_bufs);
    rc |= dalloc(c, &d_adj_off, nn + 1, c->topo_bufs);
    rc |= dalloc(c, &d_adj, std::max(na, 1ll), c->topo_bufs);
    rc |= dalloc(c, &d_stack, 4 * std::max(nn, 1ll), c->topo_bufs);
    rc |= dalloc(c, &d_status, 2, c->topo_bufs);
    rc |= dalloc(c, &d_cnt, 3 * (size_t(n) + 1), c->topo_bufs);
    rc |= dalloc(c, &d_sums, 3 * (size_t(tiles) + 1), c->topo_bufs);
    if (rc) { free_all(c->topo_bufs); return fail(c, GRB_ENOMEM, "topology scratch"); }
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, h2d(d_node_off, t->node_off, sizeof(int) * (n + 1)));
    GRB_CUDA(c, h2d(d_pos, t->pos, sizeof(int) * nn));
    GRB_CUDA(c, h2d(d_adj_off, t->adj_off, sizeof(int) * (nn + 1)));
    GRB_CUDA(c, h2d(d_adj, t->adj, sizeof(int) * na));
    GRB_CUDA(c, cudaMemsetAsync(d_status, 0, 2 * sizeof(int), c->stream));
    TopoBuild B{n, c->T.X, c->T.Y, c->T.L, nn, na, d_node_off, d_pos, d_adj_off, d_adj,
                {d_cnt, d_cnt + n + 1, d_cnt + 2 * (n + 1)}};
    B.stack = d_stack;
    B.seen = d_stack + 3 * nn;
    B.status = d_status;
    const int grid = std::max(1, (n + 255) / 256);
    if (n) k_topo_count<<<grid, 256, 0, c->stream>>>(B);
    for (int k = 0; k < 3; ++k) {
        long long* sums = d_sums + k * (tiles + 1);
        if (n) k_scan_tiles<<<tiles, 256, 0, c->stream>>>(B.cnt[k], n, sums);
        k_scan_sums<<<1, 1024, 0, c->stream>>>(sums, tiles);
        k_scan_add<<<n / 256 + 1, 256, 0, c->stream>>>(B.cnt[k], n, sums, tiles);
    }
    c->launches += (n ? 1 : 0) + 3 * (n ? 3 : 2);
    GRB_CUDA(c, cudaGetLastError());
    long long tot[3] = {0, 0, 0};
    int status[2] = {0, 0};
    for (int k = 0; k < 3; ++k)
        GRB_CUDA(c, cudaMemcpyAsync(tot + k, B.cnt[k] + n, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    static const char* what[] = {"", "tree adjacency outside its net", "tree node outside the grid",
                                 "adjacency is not a tree on the net's nodes"};
    if (status[0]) {
        free_all(c->topo_bufs);
        c->n_nets = 0;
        return fail(c, GRB_EINVAL, std::string(what[status[0]]) + " (net " + std::to_string(status[1]) + ")");
    }
    if (tot[0] > INT_MAX || 2 * tot[1] > INT_MAX || 2 * tot[2] > INT_MAX) {
        free_all(c->topo_bufs);
        return fail(c, GRB_EINVAL, "geometry exceeds 2^31 entries");
    }
    const long long need[6] = {n, nn, rw, tot[0], tot[1], tot[2]};
    if (int e = net_buffers(c, need)) { free_all(c->topo_bufs); return e; }
    GRB_CUDA(c, cudaMemcpyAsync(c->node_off, d_node_off, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, c->stream));
    GRB_CUDA(c, h2d(c->route_off, t->route_off, sizeof(long long) * (n + 1)));
    GRB_CUDA(c, cudaMemsetAsync(c->routes, 0, sizeof(int) * std::max<long long>(rw, 1), c->stream));
    B.nodes = c->nodes;
    B.parents = c->parents;
    B.point_off = c->point_off; B.points = c->points;
    B.hseg_off = c->hseg_off; B.hsegs = c->hsegs;
    B.vseg_off = c->vseg_off; B.vsegs = c->vsegs;
    if (n) {
        GRB_CUDA(c, cudaMemsetAsync(B.seen, 0, sizeof(int) * std::max(nn, 1ll), c->stream));
        k_topo_fill<<<grid, 256, 0, c->stream>>>(B);
        c->launches += 1;
    } else {
        GRB_CUDA(c, cudaMemsetAsync(c->point_off, 0, sizeof(int), c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->hseg_off, 0, sizeof(int), c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->vseg_off, 0, sizeof(int), c->stream));
    }
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    free_all(c->topo_bufs);
    if (status[0]) {
        c->n_nets = 0;
        return fail(c, GRB_EINVAL, std::string(what[status[0]]) + " (net " + std::to_string(status[1]) + ")");
    }
    return validate_net_store(c, n, int(nn), rw, int(tot[0]), int(tot[1]), int(tot[2]));
}

// Chunk of the text copied to the host per sink call.
constexpr long long kOutChunk = 64ll << 20;

int grb_format_out(grb_ctx* c, const grb_out_records* rec, int64_t* bytes) {
    if (!c || !rec || rec->n < 0 || !rec->name_off || !rec->pin_off || !rec->extra_off || !rec->sub_off || !bytes)
        return c ? fail(c, GRB_EINVAL, "bad output records") : GRB_EINVAL;
    if (c->out_pending) return fail(c, GRB_EINVAL, "the previous text has not been drained (grb_drain_out)");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = rec->n;
    if (rec->name_off[0] != 0 || rec->pin_off[0] != 0 || rec->extra_off[0] != 0 || rec->sub_off[0] != 0)
        return fail(c, GRB_EINVAL, "offsets must start at 0");
    const long long nc = rec->name_off[n], np = rec->pin_off[n], ne = rec->extra_off[n], ns = rec->sub_off[n];
    if (nc < 0 || np < 0 || ne < 0 || ns < 0) return fail(c, GRB_EINVAL, "negative totals");
    for (int r = 0; r < n; ++r)
        if (rec->name_off[r + 1] < rec->name_off[r] || rec->pin_off[r + 1] < rec->pin_off[r] ||
            rec->extra_off[r + 1] < rec->extra_off[r] || rec->sub_off[r + 1] < rec->sub_off[r])
            return fail(c, GRB_EINVAL, "offsets must be non-decreasing");
    if ((nc && !rec->names) || (np && !rec->pins) || (ne && !rec->extra) || (ns && (!rec->subnets || !rec->sub_phase2)))
        return fail(c, GRB_EINVAL, "record arrays missing");
    if (ns && !c->routes) return fail(c, GRB_EINVAL, "no nets uploaded");
    // The drain (possibly on another host thread, beside stage work on the
    // context's stream) allocates and frees nothing: stream, events and the
    // pinned chunk buffers are made here.
    if (!c->out_stream) {
        GRB_CUDA(c, cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
        GRB_CUDA(c, cudaEventCreateWithFlags(&c->out_ready, cudaEventDisableTiming));
        // Blocking events: the draining thread sleeps instead of spinning on a
        // core the caller's pipeline may need.
        for (cudaEvent_t& e : c->out_chunk_ev)
            GRB_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming | cudaEventBlockingSync));
    }
    for (char*& h : c->out_host)
        if (!h && cudaMallocHost(&h, size_t(kOutChunk)) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GRB_ENOMEM, "pinned output buffers");
        }
    free_all(c->out_bufs);
    long long* d_name_off = nullptr, *d_bytes = nullptr, *d_sums = nullptr;
    char* d_names = nullptr;
    int *d_pin_off = nullptr, *d_pins = nullptr, *d_extra_off = nullptr, *d_extra = nullptr, *d_sub_off = nullptr,
        *d_subnets = nullptr, *d_status = nullptr;
    unsigned char* d_phase2 = nullptr;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    int rc = 0;
    rc |= dalloc(c, &d_name_off, n + 1, c->out_bufs);
    rc |= dalloc(c, &d_names, std::max(nc, 1ll), c->out_bufs);
    rc |= dalloc(c, &d_pin_off, n + 1, c->out_bufs);
    rc |= dalloc(c, &d_pins, std::max(np, 1ll), c->out_bufs);
    rc |= dalloc(c, &d_extra_off, n + 1, c->out_bufs);
    rc |= dalloc(c, &d_extra, std::max(ne, 1ll), c->out_bufs);
    rc |= dalloc(c, &d_sub_off, n + 1, c->out_bufs);
    rc |= dalloc(c, &d_subnets, std::max(ns, 1ll), c->out_bufs);
    rc |= dalloc(c, &d_phase2, std::max(ns, 1ll), c->out_bufs);
    rc |= dalloc(c, &d_bytes, n + 1, c->out_bufs);
    rc |= dalloc(c, &d_sums, tiles + 1, c->out_bufs);
    rc |= dalloc(c, &d_status, 2, c->out_bufs);
    if (rc) { free_all(c->out_bufs); return fail(c, GRB_ENOMEM, "output records"); }
    auto h2d = [&](void* dst, const void* src, size_t b) {
        return b ? cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, h2d(d_name_off, rec->name_off, 8 * (size_t(n) + 1)));
    GRB_CUDA(c, h2d(d_names, rec->names, size_t(nc)));
    GRB_CUDA(c, h2d(d_pin_off, rec->pin_off, 4 * (size_t(n) + 1)));
    GRB_CUDA(c, h2d(d_pins, rec->pins, 4 * size_t(np)));
    GRB_CUDA(c, h2d(d_extra_off, rec->extra_off, 4 * (size_t(n) + 1)));
    GRB_CUDA(c, h2d(d_extra, rec->extra, 4 * size_t(ne)));
    GRB_CUDA(c, h2d(d_sub_off, rec->sub_off, 4 * (size_t(n) + 1)));
    GRB_CUDA(c, h2d(d_subnets, rec->subnets, 4 * size_t(ns)));
    GRB_CUDA(c, h2d(d_phase2, rec->sub_phase2, size_t(ns)));
    GRB_CUDA(c, cudaMemsetAsync(d_status, 0, 2 * sizeof(int), c->stream));
    OutRecords R{n, c->T.X, c->T.Y, d_name_off, d_names, d_pin_off, d_pins, d_extra_off, d_extra, d_sub_off,
                 d_subnets, d_phase2, c->route_off, c->routes, c->F.route2_off, c->F.routes2, d_bytes, nullptr,
                 d_status, c->n_nets};
    if (!c->F.routes2) R.route2_off = nullptr;
    const int blocks = std::max(1, (n + 7) / 8);  // 8 warps per CTA
    if (n) k_out_count<<<blocks, 256, 0, c->stream>>>(R);
    if (n) k_scan_tiles<<<tiles, 256, 0, c->stream>>>(d_bytes, n, d_sums);
    k_scan_sums<<<1, 1024, 0, c->stream>>>(d_sums, tiles);
    k_scan_add<<<n / 256 + 1, 256, 0, c->stream>>>(d_bytes, n, d_sums, tiles);
    c->launches += (n ? 2 : 0) + 2;
    GRB_CUDA(c, cudaGetLastError());
    long long total = 0;
    int status[2] = {0, 0};
    GRB_CUDA(c, cudaMemcpyAsync(&total, d_bytes + n, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (status[0]) {
        free_all(c->out_bufs);
        return fail(c, GRB_EINVAL, "record " + std::to_string(status[1]) + ": subnet id or its route words invalid");
    }
    if (total > c->out_text_cap) {
        if (c->out_text) cudaFree(c->out_text);
        c->out_text = nullptr;
        c->out_text_cap = 0;
        if (cudaMalloc(&c->out_text, size_t(std::max(total, 1ll))) != cudaSuccess) {
            cudaGetLastError();
            free_all(c->out_bufs);
            return fail(c, GRB_ENOMEM, "output text");
        }
        c->out_text_cap = total;
    }
    R.text = c->out_text;
    if (n) k_out_write<<<blocks, 256, 0, c->stream>>>(R);
    c->launches += n ? 1 : 0;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaEventRecord(c->out_ready, c->stream));
    c->out_bytes = total;
    c->out_pending = true;
    *bytes = total;
    return GRB_OK;
}

int grb_drain_out(grb_ctx* c, grb_out_sink sink, void* user) {
    if (!c || !sink) return c ? fail(c, GRB_EINVAL, "no sink") : GRB_EINVAL;
    if (!c->out_pending) return GRB_OK;
    GRB_CUDA(c, cudaSetDevice(c->device));
    GRB_CUDA(c, cudaStreamWaitEvent(c->out_stream, c->out_ready, 0));
    const long long total = c->out_bytes;
    const long long chunks = (total + kOutChunk - 1) / kOutChunk;
    auto issue = [&](long long k) {
        const long long off = k * kOutChunk, len = std::min(kOutChunk, total - off);
        cudaError_t e = cudaMemcpyAsync(c->out_host[k & 1], c->out_text + off, size_t(len), cudaMemcpyDeviceToHost,
                                        c->out_stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->out_chunk_ev[k & 1], c->out_stream);
        return e;
    };
    if (chunks) GRB_CUDA(c, issue(0));
    int rc = GRB_OK;
    for (long long k = 0; k < chunks; ++k) {
        GRB_CUDA(c, cudaEventSynchronize(c->out_chunk_ev[k & 1]));
        if (k + 1 < chunks) GRB_CUDA(c, issue(k + 1));  // the other buffer was consumed at step k - 1
        const long long len = std::min(kOutChunk, total - k * kOutChunk);
        if (sink(c->out_host[k & 1], len, user) != 0) { rc = fail(c, GRB_EINVAL, "the output sink failed"); break; }
    }
    // (every copy has been waited for through its chunk event)
    c->out_pending = false;
    return rc;
}

int grb_remove_routes(grb_ctx* c, const int32_t* ids, int32_t n, const uint8_t* phase2) {
    if (!c || n < 0 || (n && (!ids || !phase2))) return c ? fail(c, GRB_EINVAL, "bad removal list") : GRB_EINVAL;
    if (!c->routes) return fail(c, GRB_EINVAL, "no nets uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (n == 0) return GRB_OK;
    for (int k = 0; k < n; ++k) {
        if (ids[k] < 0 || ids[k] >= c->n_nets) return fail(c, GRB_EINVAL, "net id out of range (item " + std::to_string(k) + ")");
        if (phase2[k] && (c->flt_n != c->n_nets || c->h_route2_off[ids[k] + 1] == c->h_route2_off[ids[k]]))
            return fail(c, GRB_EINVAL, "net " + std::to_string(ids[k]) + " has no phase-two routes");
    }
    int* d_ids = nullptr;
    unsigned char* d_ph = nullptr;
    if (cudaMalloc(&d_ids, sizeof(int) * n) != cudaSuccess || cudaMalloc(&d_ph, size_t(n)) != cudaSuccess) {
        cudaGetLastError();
        if (d_ids) cudaFree(d_ids);
        return fail(c, GRB_ENOMEM, "removal list");
    }
    GRB_CUDA(c, cudaMemcpyAsync(d_ids, ids, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(d_ph, phase2, size_t(n), cudaMemcpyHostToDevice, c->stream));
    Plan P = make_plan(c);
    Plan P2 = c->F.routes2 ? make_plan2(c) : P;
    k_maze_remove<<<(n + 127) / 128, 128, 0, c->stream>>>(c->T, P, P2, RemoveList{d_ids, d_ph, n});
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_ids);
    cudaFree(d_ph);
    return check_device_error(c);
}

int grb_routing_score(grb_ctx* c, double* score) {
    if (!c || !score) return c ? fail(c, GRB_EINVAL, "null score") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (!c->score_partials && cudaMalloc(&c->score_partials, sizeof(double) * kScoreBlocks) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GRB_ENOMEM, "score partials");
    }
    k_maze_score<<<kScoreBlocks, kScoreThreads, 0, c->stream>>>(c->T, c->score_partials);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    std::vector<double> host(kScoreBlocks);
    GRB_CUDA(c, cudaMemcpyAsync(host.data(), c->score_partials, sizeof(double) * kScoreBlocks, cudaMemcpyDeviceToHost,
                                c->stream));
    double wl = 0;
    unsigned long long vias = 0;
    GRB_CUDA(c, cudaMemcpyAsync(&wl, c->T.wirelength, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(&vias, c->T.vias, sizeof(vias), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    double s = wl * c->T.unit_wire + static_cast<double>(static_cast<long long>(vias)) * c->T.unit_via;
    for (double v : host) s += v;
    *score = s;
    return GRB_OK;
}

int grb_checkpoint(grb_ctx* c) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (!c->ckpt_demand && cudaMalloc(&c->ckpt_demand, sizeof(int) * size_t(c->T.cells)) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GRB_ENOMEM, "checkpoint");
    }
    GRB_CUDA(c, cudaMemcpyAsync(c->ckpt_demand, c->T.demand, sizeof(int) * size_t(c->T.cells), cudaMemcpyDeviceToDevice,
                                c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(&c->ckpt_wirelength, c->T.wirelength, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(&c->ckpt_vias, c->T.vias, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_restore(grb_ctx* c) {
    if (!c) return GRB_EINVAL;
    if (!c->ckpt_demand) return fail(c, GRB_EINVAL, "no checkpoint");
    GRB_CUDA(c, cudaSetDevice(c->device));
    GRB_CUDA(c, cudaMemcpyAsync(c->T.demand, c->ckpt_demand, sizeof(int) * size_t(c->T.cells), cudaMemcpyDeviceToDevice,
                                c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(c->T.wirelength, &c->ckpt_wirelength, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(c->T.vias, &c->ckpt_vias, sizeof(unsigned long long), cudaMemcpyHostToDevice, c->stream));
    // Every cost is recomputed at the next refresh (the reference clears
    // costs_initialized, maze_quality.cuh:100).
    k_mark_all_dirty<<<(c->T.cells + 255) / 256, 256, 0, c->stream>>>(c->T);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_topology_sizes(grb_ctx* c, int64_t* sizes) {
    if (!c || !sizes) return c ? fail(c, GRB_EINVAL, "null") : GRB_EINVAL;
    for (int k = 0; k < 4; ++k) sizes[k] = c->topo_sizes[k];
    return GRB_OK;
}

int grb_read_topology(grb_ctx* c, int32_t* node_off, int32_t* nodes, int32_t* parents, int32_t* point_off,
                      int32_t* points, int32_t* hseg_off, int32_t* hsegs, int32_t* vseg_off, int32_t* vsegs) {
    if (!c) return GRB_EINVAL;
    if (c->topo_sizes[0] < 0) return fail(c, GRB_EINVAL, "no nets");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const size_t n1 = size_t(c->n_nets) + 1;
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return dst && bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, d2h(node_off, c->node_off, 4 * n1));
    GRB_CUDA(c, d2h(nodes, c->nodes, 4 * size_t(c->topo_sizes[0])));
    GRB_CUDA(c, d2h(parents, c->parents, 4 * size_t(c->topo_sizes[0])));
    GRB_CUDA(c, d2h(point_off, c->point_off, 4 * n1));
    GRB_CUDA(c, d2h(points, c->points, 4 * size_t(c->topo_sizes[1])));
    GRB_CUDA(c, d2h(hseg_off, c->hseg_off, 4 * n1));
    GRB_CUDA(c, d2h(hsegs, c->hsegs, 8 * size_t(c->topo_sizes[2])));
    GRB_CUDA(c, d2h(vseg_off, c->vseg_off, 4 * n1));
    GRB_CUDA(c, d2h(vsegs, c->vsegs, 8 * size_t(c->topo_sizes[3])));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_set_wire_cost_mode(grb_ctx* c, int32_t integer_wire) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    c->T.int_wire = integer_wire ? 1 : 0;
    // Every wire cost changes: the next refresh recomputes all cells and tracks.
    const int n = std::max(c->T.words, c->T.n_groups);
    k_mark_all_dirty<<<(n + 255) / 256, 256, 0, c->stream>>>(c->T);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_upload_zshape(grb_ctx* c, const grb_zshape_trees* t) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!t || !t->node_off) return fail(c, GRB_EINVAL, "Z-shape tree offsets missing");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const Tables& T = c->T;
    const int n = c->n_nets, XY = T.XY;
    const int N = std::max(T.X, T.Y), LAYER = T.L + 1;
    const long long NN = (long long)N * N, LNN = LAYER * NN;
    if (16 * LNN >= (1ll << 31)) return fail(c, GRB_EINVAL, "Z-shape planes exceed 32-bit indexing");
    if (t->node_off[0] != 0) return fail(c, GRB_EINVAL, "Z-shape offsets must start at 0");
    for (int i = 0; i < n; ++i) if (t->node_off[i + 1] < t->node_off[i]) return fail(c, GRB_EINVAL, "Z-shape offsets must be non-decreasing");
    const long long nn = t->node_off[n];
    if (nn && (!t->coord || !t->child)) return fail(c, GRB_EINVAL, "Z-shape tree arrays missing");
    std::vector<int> pos(nn), pin(nn);
    std::vector<int4> box(std::max(n, 1));
    for (int id = 0; id < n; ++id) {
        const int nb = t->node_off[id], cnt = t->node_off[id + 1] - nb;
        int4 bb = make_int4(T.X, 0, T.Y, 0);
        for (int i = 0; i < cnt; ++i) {
            const int cd = t->coord[nb + i];
            if (cd < 0 || cd / XY > T.L) return fail(c, GRB_EINVAL, "Z-shape node outside the grid");
            const int l = cd / XY, x = cd % XY / T.Y, y = cd % T.Y;
            pos[nb + i] = x * N + y;                 // zshape_topology.hpp:105
            pin[nb + i] = l < T.L ? l + 1 : -1;      // :106-109
            bb.x = std::min(bb.x, x); bb.y = std::max(bb.y, x);
            bb.z = std::min(bb.z, y); bb.w = std::max(bb.w, y);
            for (int j = 0; j < 3; ++j) {
                const int ch = t->child[3 * (size_t(nb) + i) + j];
                if (ch != -1 && (ch <= i || ch >= cnt)) return fail(c, GRB_EINVAL, "Z-shape children must follow their parent in preorder");
            }
        }
        if (!cnt) bb = make_int4(0, 0, 0, 0);
        box[id] = bb;
    }
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    const bool planes = c->Z.map != nullptr && c->Z.LNN == LNN;
    std::vector<void*> keep;
    if (planes) {  // keep the (large) planes, replace the per-node arrays
        for (void* p : c->z_bufs)
            if (p == c->Z.map || p == c->Z.prev) keep.push_back(p);
            else cudaFree(p);
        c->z_bufs = keep;
    } else {
        free_all(c->z_bufs);
    }
    ZTrees Z = c->Z;
    int *noff, *dpos, *dpin, *dch;
    int4* dbox;
    int rc = 0;
    rc |= dalloc(c, &noff, n + 1, c->z_bufs);
    rc |= dalloc(c, &dpos, nn, c->z_bufs);
    rc |= dalloc(c, &dpin, nn, c->z_bufs);
    rc |= dalloc(c, &dch, 3 * nn, c->z_bufs);
    rc |= dalloc(c, &dbox, std::max(n, 1), c->z_bufs);
    if (!planes) {
        rc |= dalloc(c, &Z.map, size_t(6) * LNN, c->z_bufs);
        rc |= dalloc(c, &Z.prev, size_t(16) * LNN, c->z_bufs);
    }
    if (rc) { free_all(c->z_bufs); c->Z = ZTrees{}; c->z_n = -1; return GRB_ENOMEM; }
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, h2d(noff, t->node_off, 4 * size_t(n + 1)));
    GRB_CUDA(c, h2d(dpos, pos.data(), 4 * size_t(nn)));
    GRB_CUDA(c, h2d(dpin, pin.data(), 4 * size_t(nn)));
    GRB_CUDA(c, h2d(dch, t->child, 12 * size_t(nn)));
    GRB_CUDA(c, h2d(dbox, box.data(), sizeof(int4) * box.size()));
    if (!planes) {
        GRB_CUDA(c, cudaMemsetAsync(Z.map, 0, sizeof(int) * 6 * LNN, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(Z.prev, 0, sizeof(int) * 16 * LNN, c->stream));
    }
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    Z.node_off = noff; Z.pos = dpos; Z.pin = dpin; Z.child = dch;
    Z.N = N; Z.LAYER = LAYER; Z.D = T.DIR ^ 1; Z.NN = NN; Z.LNN = LNN;
    c->Z = Z;
    c->z_box = dbox;
    c->z_n = n;
    c->h_z_node_off.assign(t->node_off, t->node_off + n + 1);
    ++c->z_version;
    return GRB_OK;
}

int grb_plan_bbox_batches(grb_ctx* c, const int32_t* bbox, int32_t max_batch, int32_t* n_batches) {
    if (!c) return GRB_EINVAL;
    if (max_batch < 1 || max_batch > kMaxBoxBatch) return fail(c, GRB_EINVAL, "max_batch must be in [1, 256]");
    if (!bbox && c->z_n != c->n_nets) return fail(c, GRB_EINVAL, "no boxes given and no Z-shape trees uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = c->plan_n, G = c->n_batches;
    if (n == 0) { if (n_batches) *n_batches = 0; return GRB_OK; }
    std::vector<void*> tmpb;
    int4* box = c->z_box;
    if (bbox) {
        for (int i = 0; i < c->n_nets; ++i) {
            const int* b = bbox + 4 * size_t(i);
            if (b[0] < 0 || b[0] > b[1] || b[1] >= c->T.X || b[2] < 0 || b[2] > b[3] || b[3] >= c->T.Y)
                return fail(c, GRB_EINVAL, "net box outside the grid");
        }
        if (dalloc(c, &box, c->n_nets, tmpb)) return GRB_ENOMEM;
        GRB_CUDA(c, cudaMemcpyAsync(box, bbox, sizeof(int4) * c->n_nets, cudaMemcpyHostToDevice, c->stream));
    }
    // Scratch kept in the context (grow-only): allocating and freeing it on
    // every call costs more than the refinement itself.
    if (n > c->box_cap_n || G > c->box_cap_g) {
        free_all(c->box_bufs);
        c->box_cap_n = c->box_cap_g = 0;
        const int cn = std::max(n, c->box_cap_n), cg = std::max(G, c->box_cap_g);
        int rc = 0;
        rc |= dalloc(c, &c->box_ka, cn, c->box_bufs); rc |= dalloc(c, &c->box_kb, cn, c->box_bufs);
        rc |= dalloc(c, &c->box_pend, cn, c->box_bufs); rc |= dalloc(c, &c->box_tmp, cn, c->box_bufs);
        rc |= dalloc(c, &c->box_bsize, cn, c->box_bufs); rc |= dalloc(c, &c->box_bofs, cn, c->box_bufs);
        rc |= dalloc(c, &c->box_rounds, cg, c->box_bufs); rc |= dalloc(c, &c->box_first, cg, c->box_bufs);
        rc |= dalloc(c, &c->box_off, cn + 1, c->box_bufs);
        if (rc) { free_all(c->box_bufs); free_all(tmpb); return GRB_ENOMEM; }
        c->box_cap_n = cn;
        c->box_cap_g = cg;
    }
    unsigned long long *ka = c->box_ka, *kb = c->box_kb;
    int *pend = c->box_pend, *tmp = c->box_tmp, *bsize = c->box_bsize, *bofs = c->box_bofs;
    int *rounds = c->box_rounds, *first = c->box_first, *off_new = c->box_off;
    auto run = [&]() -> int {
        k_bbox_refine<<<G, kBoxThreads, 0, c->stream>>>(c->ids, c->batch_off, box, ka, kb, pend, tmp, bsize, rounds,
                                                        max_batch);
        c->launches += 1;
        GRB_CUDA(c, cudaGetLastError());
        std::vector<int> hr(G), hf(G);
        GRB_CUDA(c, cudaMemcpyAsync(hr.data(), rounds, 4 * size_t(G), cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        int total = 0;
        for (int g = 0; g < G; ++g) { hf[g] = total; total += hr[g]; }
        GRB_CUDA(c, cudaMemcpyAsync(first, hf.data(), 4 * size_t(G), cudaMemcpyHostToDevice, c->stream));
        k_bbox_scatter<<<G, kBoxThreads, 0, c->stream>>>(c->batch_off, tmp, bsize, rounds, first, bofs, c->ids, off_new);
        c->launches += 1;
        GRB_CUDA(c, cudaGetLastError());
        std::vector<int> h(total + 1);
        GRB_CUDA(c, cudaMemcpyAsync(h.data(), off_new, 4 * size_t(total), cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        h[total] = n;
        if (total > c->plan_cap) return fail(c, GRB_EINVAL, "more batches than plan capacity");
        GRB_CUDA(c, cudaMemcpyAsync(c->batch_off, h.data(), 4 * size_t(total + 1), cudaMemcpyHostToDevice, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->h_batch_off = h;
        c->n_batches = total;
        ++c->plan_version;
        if (n_batches) *n_batches = total;
        return GRB_OK;
    };
    const int r = run();
    cudaStreamSynchronize(c->stream);
    free_all(tmpb);
    return r;
}

int grb_upload_geometry(grb_ctx* c, const int32_t* point_off, const int32_t* points, const int32_t* hseg_off,
                        const int32_t* hsegs, const int32_t* vseg_off, const int32_t* vsegs) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!point_off || !hseg_off || !vseg_off) return fail(c, GRB_EINVAL, "geometry offsets missing");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n_nets, XY = c->T.XY;
    const int* offs[3] = {point_off, hseg_off, vseg_off};
    const int* data[3] = {points, hsegs, vsegs};
    const int width[3] = {1, 2, 2};
    for (int k = 0; k < 3; ++k) {
        if (offs[k][0] != 0) return fail(c, GRB_EINVAL, "geometry offsets must start at 0");
        for (int i = 0; i < n; ++i) if (offs[k][i + 1] < offs[k][i]) return fail(c, GRB_EINVAL, "geometry offsets must be non-decreasing");
        if (offs[k][n] && !data[k]) return fail(c, GRB_EINVAL, "geometry data missing");
        for (long long q = 0; q < (long long)offs[k][n] * width[k]; ++q)
            if (data[k][q] < 0 || data[k][q] >= XY) return fail(c, GRB_EINVAL, "batching geometry outside the grid");
    }
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    free_all(c->geom_bufs);
    int* d[6];
    int rc = 0;
    rc |= dalloc(c, &d[0], n + 1, c->geom_bufs);
    rc |= dalloc(c, &d[1], point_off[n], c->geom_bufs);
    rc |= dalloc(c, &d[2], n + 1, c->geom_bufs);
    rc |= dalloc(c, &d[3], 2 * size_t(hseg_off[n]), c->geom_bufs);
    rc |= dalloc(c, &d[4], n + 1, c->geom_bufs);
    rc |= dalloc(c, &d[5], 2 * size_t(vseg_off[n]), c->geom_bufs);
    if (rc) { free_all(c->geom_bufs); return GRB_ENOMEM; }
    for (int k = 0; k < 3; ++k) {
        GRB_CUDA(c, cudaMemcpyAsync(d[2 * k], offs[k], sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->stream));
        if (offs[k][n])
            GRB_CUDA(c, cudaMemcpyAsync(d[2 * k + 1], data[k], sizeof(int) * width[k] * size_t(offs[k][n]),
                                        cudaMemcpyHostToDevice, c->stream));
    }
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->point_off = d[0]; c->points = d[1]; c->hseg_off = d[2]; c->hsegs = d[3]; c->vseg_off = d[4]; c->vsegs = d[5];
    return GRB_OK;
}

int grb_upload_flt(grb_ctx* c, const grb_flt_dags* d) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!d || !d->node_off || !d->edge_off || !d->route2_off) return fail(c, GRB_EINVAL, "FLT DAG offsets missing");
    if (c->T.L != kFltLayers - 1) return fail(c, GRB_EINVAL, "the FLT stage needs 9 routing layers (MAX_LAYER 10)");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const Tables& T = c->T;
    const int n = c->n_nets, XY = T.XY;
    if (d->node_off[0] != 0 || d->edge_off[0] != 0 || d->route2_off[0] != 0) return fail(c, GRB_EINVAL, "FLT offsets must start at 0");
    for (int i = 0; i < n; ++i)
        if (d->node_off[i + 1] < d->node_off[i] || d->edge_off[i + 1] < d->edge_off[i] || d->route2_off[i + 1] < d->route2_off[i])
            return fail(c, GRB_EINVAL, "FLT offsets must be non-decreasing");
    const long long nn = d->node_off[n], ne = d->edge_off[n];
    if ((nn && (!d->coord || !d->depth || !d->children || !d->parent_end)) || (ne && (!d->edge_parent || !d->edge_source_slot)))
        return fail(c, GRB_EINVAL, "FLT DAG arrays missing");
    // Host validation (every index the kernels dereference) and the derived
    // per-node arrays: global child offsets, depth-sorted order, level offsets.
    std::vector<int> child_off(size_t(nn) + 1), order(nn), eslot(ne), lvl_off(n + 1, 0), level, width(n, 0);
    long long children = 0;
    for (int id = 0; id < n; ++id) {
        const int nb = d->node_off[id], N = d->node_off[id + 1] - nb;
        const int eb = d->edge_off[id], E = d->edge_off[id + 1] - eb;
        lvl_off[id] = int(level.size());
        if (N == 0) {
            if (E) return fail(c, GRB_EINVAL, "FLT edges without nodes");
            continue;
        }
        if (N >= (1ll << 31) / 100 - 1) return fail(c, GRB_EINVAL, "FLT DAG too large for packed candidate ids");
        int maxd = 0;
        for (int i = 0; i < N; ++i) {
            const int g = nb + i;
            const int cd = d->coord[g], dp = d->depth[g], ch = d->children[g];
            if (cd < 0 || cd / XY > kFltLayers - 1) return fail(c, GRB_EINVAL, "FLT node outside the grid");
            if (dp < 0 || dp >= 5000) return fail(c, GRB_EINVAL, "FLT depth out of range");  // flt_topology.hpp:58
            if (ch < 0 || ch > kFltMaxChildren) return fail(c, GRB_EINVAL, "FLT node with more than 6 child slots");
            const int pb = i ? d->parent_end[g - 1] : 0, pe = d->parent_end[g];
            if (pe < pb || pe > E) return fail(c, GRB_EINVAL, "FLT parent ranges inconsistent");
            child_off[g] = int(children);
            children += ch;
            maxd = std::max(maxd, dp);
        }
        if (d->parent_end[nb + N - 1] != E) return fail(c, GRB_EINVAL, "FLT parent ranges do not cover the edges");
        for (int i = 0; i < N; ++i) {
            const int g = nb + i;
            const int pb = i ? d->parent_end[g - 1] : 0, pe = d->parent_end[g];
            const int cx = d->coord[g] % XY / T.Y, cy = d->coord[g] % T.Y;
            for (int e = eb + pb; e < eb + pe; ++e) {
                const int p = d->edge_parent[e], src = d->edge_source_slot[e];
                if (p < 0 || p >= N || src < 0 || src / 10 != i) return fail(c, GRB_EINVAL, "FLT edge endpoints inconsistent");
                if (d->depth[nb + p] >= d->depth[g]) return fail(c, GRB_EINVAL, "FLT parent not shallower than child");
                if (src % 10 >= d->children[nb + p]) return fail(c, GRB_EINVAL, "FLT child slot out of range");
                const int px = d->coord[nb + p] % XY / T.Y, py = d->coord[nb + p] % T.Y;
                if (px != cx && py != cy) return fail(c, GRB_EINVAL, "FLT edge is not straight");
                eslot[e] = src;
            }
        }
        std::vector<int> cnt(maxd + 2, 0);
        for (int i = 0; i < N; ++i) ++cnt[d->depth[nb + i] + 1];
        for (int q = 0; q <= maxd; ++q) width[id] = std::max(width[id], cnt[q + 1]);
        for (int q = 0; q <= maxd; ++q) cnt[q + 1] += cnt[q];
        for (int q = 0; q <= maxd + 1; ++q) level.push_back(cnt[q]);
        for (int i = 0; i < N; ++i) order[nb + cnt[d->depth[nb + i]]++] = i;  // stable by index
    }
    lvl_off[n] = int(level.size());
    if (children >= (1ll << 31) / kFltLayers) return fail(c, GRB_EINVAL, "too many FLT child slots");
    child_off[nn] = int(children);
    for (int i = 0; i < n; ++i) {
        if (d->node_off[i + 1] > d->node_off[i] && d->route2_off[i + 1] - d->route2_off[i] < 1)
            return fail(c, GRB_EINVAL, "FLT net without phase-two route storage");
    }
    const long long rw = d->route2_off[n];
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    free_all(c->flt_bufs);
    c->flt_n = -1;
    Flt F{};
    int *node_off, *edge_off, *lvl, *levelp, *coord, *ch, *coff, *pend, *ord, *epar, *es, *lo, *bc, *r2;
    long long* r2off;
    double *costs, *ce;
    unsigned long long *packed, *best;
    int rc = 0;
    std::vector<void*>& B = c->flt_bufs;
    rc |= dalloc(c, &node_off, n + 1, B); rc |= dalloc(c, &edge_off, n + 1, B);
    rc |= dalloc(c, &lvl, n + 1, B); rc |= dalloc(c, &levelp, level.size(), B);
    rc |= dalloc(c, &r2off, n + 1, B); rc |= dalloc(c, &r2, std::max<long long>(rw, 1), B);
    rc |= dalloc(c, &coord, nn, B); rc |= dalloc(c, &ch, nn, B); rc |= dalloc(c, &coff, nn + 1, B);
    rc |= dalloc(c, &pend, nn, B); rc |= dalloc(c, &ord, nn, B); rc |= dalloc(c, &lo, nn, B);
    rc |= dalloc(c, &epar, ne, B); rc |= dalloc(c, &es, ne, B);
    rc |= dalloc(c, &costs, size_t(nn) * kFltLayers, B);
    rc |= dalloc(c, &packed, size_t(children) * kFltLayers, B);
    rc |= dalloc(c, &best, size_t(children) * kFltLayers, B);
    rc |= dalloc(c, &ce, size_t(ne) * 81, B); rc |= dalloc(c, &bc, size_t(ne) * 81, B);
    if (rc) { free_all(B); return GRB_ENOMEM; }
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) : cudaSuccess;
    };
    GRB_CUDA(c, h2d(node_off, d->node_off, 4 * (n + 1)));
    GRB_CUDA(c, h2d(edge_off, d->edge_off, 4 * (n + 1)));
    GRB_CUDA(c, h2d(lvl, lvl_off.data(), 4 * (n + 1)));
    GRB_CUDA(c, h2d(levelp, level.data(), 4 * level.size()));
    GRB_CUDA(c, h2d(r2off, d->route2_off, 8 * (n + 1)));
    GRB_CUDA(c, cudaMemsetAsync(r2, 0, 4 * std::max<long long>(rw, 1), c->stream));
    GRB_CUDA(c, h2d(coord, d->coord, 4 * nn));
    GRB_CUDA(c, h2d(ch, d->children, 4 * nn));
    GRB_CUDA(c, h2d(coff, child_off.data(), 4 * (nn + 1)));
    GRB_CUDA(c, h2d(pend, d->parent_end, 4 * nn));
    GRB_CUDA(c, h2d(ord, order.data(), 4 * nn));
    GRB_CUDA(c, h2d(epar, d->edge_parent, 4 * ne));
    GRB_CUDA(c, h2d(es, eslot.data(), 4 * ne));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    F.node_off = node_off; F.edge_off = edge_off; F.lvl_off = lvl; F.level = levelp; F.route2_off = r2off;
    F.coord = coord; F.children = ch; F.child_off = coff; F.pend = pend; F.order = ord;
    F.eparent = epar; F.eslot = es; F.costs = costs; F.packed = packed; F.best = best; F.lo = lo;
    F.ce = ce; F.bc = bc; F.routes2 = r2;
    c->F = F;
    c->route2_words = rw;
    c->flt_n = n;
    c->h_flt_node_off.assign(d->node_off, d->node_off + n + 1);
    c->h_flt_edge_off.assign(d->edge_off, d->edge_off + n + 1);
    c->h_route2_off.assign(d->route2_off, d->route2_off + n + 1);
    c->h_flt_width = std::move(width);
    ++c->flt_version;
    return GRB_OK;
}

int grb_set_plan(grb_ctx* c, const int32_t* ids, int32_t n, const int32_t* batch_off, int32_t nb) {
    if (!c || n < 0 || nb < 0 || (n && !ids) || !batch_off) return c ? fail(c, GRB_EINVAL, "bad plan") : GRB_EINVAL;
    if (batch_off[0] != 0 || batch_off[nb] != n) return fail(c, GRB_EINVAL, "batch offsets must span the ids");
    for (int i = 0; i < n; ++i)
        if (ids[i] < 0 || ids[i] >= c->n_nets) return fail(c, GRB_EINVAL, "net id out of range");
    int rc = ensure_plan_capacity(c, n, nb);
    if (rc) return rc;
    if (nb + 1 > c->plan_cap + 1) return fail(c, GRB_EINVAL, "more batches than nets");
    GRB_CUDA(c, cudaMemcpyAsync(c->ids, ids, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(c->batch_off, batch_off, sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, c->stream));
    c->h_batch_off.assign(batch_off, batch_off + nb + 1);
    c->plan_n = n;
    c->n_batches = nb;
    ++c->plan_version;
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_get_plan(grb_ctx* c, int32_t* ids, int32_t* batch_off, int32_t* n, int32_t* nb) {
    if (!c) return GRB_EINVAL;
    if (n) *n = c->plan_n;
    if (nb) *nb = c->n_batches;
    if (ids && c->plan_n) GRB_CUDA(c, cudaMemcpyAsync(ids, c->ids, sizeof(int) * c->plan_n, cudaMemcpyDeviceToHost, c->stream));
    if (batch_off) std::copy(c->h_batch_off.begin(), c->h_batch_off.end(), batch_off);
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

// Copies the order and builds its flat mark and query-point lists
// (k_flat_count, two scans, k_flat_fill); refuses net ids outside the
// uploaded nets.
static int build_flat_lists(grb_ctx* c, const int32_t* order, BatchState& B) {
    const int n = B.n;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    if (c->bn_cap < n || !c->order) {
        for (void** p : {(void**)&c->batch_of, (void**)&c->brank, (void**)&c->order, (void**)&c->mark_off,
                         (void**)&c->pt_off, (void**)&c->scan_sums}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        c->bn_cap = 0;
        const size_t m = std::max(n, 1);
        const size_t t = size_t(tiles) + 1;
        if (cudaMalloc(&c->batch_of, 4 * m) || cudaMalloc(&c->brank, 4 * m) || cudaMalloc(&c->order, 4 * m) ||
            cudaMalloc(&c->mark_off, 8 * (m + 1)) || cudaMalloc(&c->pt_off, 8 * (m + 1)) ||
            cudaMalloc(&c->scan_sums, 16 * t)) {
            cudaGetLastError();
            return fail(c, GRB_ENOMEM, "batching buffers");
        }
        c->bn_cap = n;
    }
    if (n) GRB_CUDA(c, cudaMemcpyAsync(c->order, order, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    B.order = c->order;
    B.batch_of = c->batch_of;
    B.rank = c->brank;
    B.mark_off = c->mark_off;
    B.pt_off = c->pt_off;
    const int grid = c->sms * 8;
    if (n) k_flat_count<<<grid, 256, 0, c->stream>>>(B, c->n_nets);
    long long* sums[2] = {c->scan_sums, c->scan_sums + tiles + 1};
    long long* arr[2] = {c->mark_off, c->pt_off};
    for (int k = 0; k < 2; ++k) {
        if (n) k_scan_tiles<<<tiles, 256, 0, c->stream>>>(arr[k], n, sums[k]);
        k_scan_sums<<<1, 1024, 0, c->stream>>>(sums[k], tiles);
        k_scan_add<<<n / 256 + 1, 256, 0, c->stream>>>(arr[k], n, sums[k], tiles);
    }
    c->launches += (n ? 1 : 0) + 2 * (n ? 3 : 2);
    GRB_CUDA(c, cudaGetLastError());
    long long tot[2] = {0, 0};
    int err[2] = {0, 0};
    GRB_CUDA(c, cudaMemcpyAsync(tot, c->mark_off + n, 8, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(tot + 1, c->pt_off + n, 8, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(err, c->T.error, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (err[0] == kEInval) {
        GRB_CUDA(c, cudaMemsetAsync(c->T.error, 0, 2 * sizeof(int), c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        return fail(c, GRB_EINVAL, "net id out of range (order position " + std::to_string(err[1]) + ")");
    }
    if (err[0]) return check_device_error(c);
    auto grow = [&](long long need, long long& cap, unsigned*& cell, unsigned short*& jj) {
        if (need <= cap) return true;
        if (cell) cudaFree(cell);
        if (jj) cudaFree(jj);
        cell = nullptr;
        jj = nullptr;
        cap = 0;
        const long long want = need + need / 8 + 1024;
        if (cudaMalloc(&cell, 4 * size_t(want)) || cudaMalloc(&jj, 2 * size_t(want))) {
            cudaGetLastError();
            return false;
        }
        cap = want;
        return true;
    };
    if (!grow(tot[0], c->mark_cap, c->mark_cell, c->mark_jj) || !grow(tot[1], c->pt_cap, c->pt_cell, c->pt_jj))
        return fail(c, GRB_ENOMEM, "batching mark lists");
    B.mark_cell = c->mark_cell; B.mark_jj = c->mark_jj;
    B.pt_cell = c->pt_cell; B.pt_jj = c->pt_jj;
    if (n) {
        k_flat_fill<<<grid, 256, 0, c->stream>>>(B);
        c->launches += 1;
        GRB_CUDA(c, cudaGetLastError());
    }
    return GRB_OK;
}

int grb_plan_batches(grb_ctx* c, const int32_t* order, int32_t n, int32_t limit, int32_t sparsity, int32_t mode,
                     int32_t* batch_of, int32_t* n_batches) {
    if (!c || n < 0 || limit < 1 || sparsity < 1 || (n && !order)) return c ? fail(c, GRB_EINVAL, "bad batching arguments") : GRB_EINVAL;
    if (mode != GRB_MODE_PLAIN && mode != GRB_MODE_GRAPH && mode != GRB_MODE_PERSISTENT)
        return fail(c, GRB_EINVAL, "unknown mode");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const size_t xy = size_t(c->T.XY);
    const size_t lm_bytes = xy * kChunkMaxWords * 4;
    const size_t pq_bytes = 2 * size_t(kChunkMax) * kChunkMaxWords * 4;
    int W = std::max(c->bW, 8);
    int rc = ensure_plan_capacity(c, n, n);
    if (rc) return rc;
    if (!c->lmask[0]) {
        if (cudaMalloc(&c->lmask[0], lm_bytes) || cudaMalloc(&c->lmask[1], lm_bytes) || cudaMalloc(&c->lmask[2], lm_bytes) ||
            cudaMalloc(&c->lmask[3], lm_bytes) || cudaMalloc(&c->lmask[4], lm_bytes) ||
            cudaMalloc(&c->ptchunk, xy * 4) ||
            cudaMalloc(&c->pred, pq_bytes) || cudaMalloc(&c->prevp, pq_bytes) || cudaMalloc(&c->bsolved, 4) ||
            cudaMalloc(&c->ncolors, 4)) {
            cudaGetLastError();
            return fail(c, GRB_ENOMEM, "batching buffers");
        }
        c->lmask_dirty = true;
    }
    BatchState B{};
    B.X = c->T.X; B.Y = c->T.Y; B.n = n; B.limit = limit; B.sparsity = sparsity;
    B.point_off = c->point_off; B.points = c->points;
    B.hseg_off = c->hseg_off; B.hsegs = c->hsegs; B.vseg_off = c->vseg_off; B.vsegs = c->vsegs;
    B.error = c->T.error; B.error_info = c->T.error_info;
    GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    if ((rc = build_flat_lists(c, order, B))) return rc;
    for (int attempt = 0; attempt < 6; ++attempt) {
        if (W != c->bW || !c->cellmask) {
            for (unsigned** p : {&c->cellmask, &c->fmask, &c->fullmask}) { if (*p) cudaFree(*p); *p = nullptr; }
            if (c->bcount) cudaFree(c->bcount);
            c->bcount = nullptr;
            c->bW = 0;
            if (cudaMalloc(&c->cellmask, xy * W * 4) || cudaMalloc(&c->fmask, 2 * size_t(kChunkMax) * W * 4) ||
                cudaMalloc(&c->fullmask, W * 4) || cudaMalloc(&c->bcount, size_t(32) * W * 4)) {
                cudaGetLastError();
                return fail(c, GRB_ENOMEM, "colour masks");
            }
            c->bW = W;
        }
        // Chunks of kChunkMax nets while the solver's shared memory fits,
        // else of half as many.
        const int CH = solve_smem_bytes<kChunkMax>(W) <= kSolveSmemLimit ? kChunkMax : kChunkMax / 2;
        const size_t smem = CH == kChunkMax ? solve_smem_bytes<kChunkMax>(W) : solve_smem_bytes<kChunkMax / 2>(W);
        if (smem > kSolveSmemLimit) return fail(c, GRB_ELIMIT, "too many batch colours");
        if (c->lmask_dirty) {
            for (unsigned* lm : c->lmask) GRB_CUDA(c, cudaMemsetAsync(lm, 0, lm_bytes, c->stream));
            GRB_CUDA(c, cudaMemsetAsync(c->ptchunk, 0, xy * 4, c->stream));
            c->lmask_dirty = false;
        }
        GRB_CUDA(c, cudaMemsetAsync(c->cellmask, 0, xy * W * 4, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->fmask, 0, 2 * size_t(kChunkMax) * W * 4, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->pred, 0, pq_bytes, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->prevp, 0, pq_bytes, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->fullmask, 0, W * 4, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->bcount, 0, size_t(32) * W * 4, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->ncolors, 0, 4, c->stream));
        GRB_CUDA(c, cudaMemsetAsync(c->bsolved, 0, 4, c->stream));
        B.W = W;
        B.cellmask = c->cellmask;
        for (int k = 0; k < 5; ++k) B.localmask[k] = c->lmask[k];
        B.ptchunk = c->ptchunk;
        B.fmask = c->fmask; B.pred = c->pred; B.prevp = c->prevp;
        B.fullmask = c->fullmask; B.count = c->bcount; B.n_colors = c->ncolors;
        B.solved = c->bsolved;
        c->lmask_dirty = true;  // until the run completes
        if ((rc = CH == kChunkMax ? launch_batching<kChunkMax>(c, B, mode, smem)
                                  : launch_batching<kChunkMax / 2>(c, B, mode, smem)))
            return rc;
        int err[2] = {0, 0};
        GRB_CUDA(c, cudaMemcpyAsync(err, c->T.error, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        if (err[0] == kELimit) {
            // Not enough colour words: retry wider (the chunk-local masks are
            // cleared at the start of the retry).
            GRB_CUDA(c, cudaMemsetAsync(c->T.error, 0, 2 * sizeof(int), c->stream));
            W *= 2;
            continue;
        }
        if (err[0]) return check_device_error(c);
        c->lmask_dirty = false;
        if (n) {
            const int C = 32 * W, tiles = (n + kRankTile - 1) / kRankTile;
            const size_t need = size_t(tiles) * C;
            if (need > c->rank_cap) {
                if (c->rank_tiles) cudaFree(c->rank_tiles);
                c->rank_tiles = nullptr;
                c->rank_cap = 0;
                if (cudaMalloc(&c->rank_tiles, 4 * need) != cudaSuccess) {
                    cudaGetLastError();
                    return fail(c, GRB_ENOMEM, "batch rank scratch");
                }
                c->rank_cap = need;
            }
            k_rank_counts<<<tiles, kRankTile, 4 * C, c->stream>>>(c->batch_of, n, C, c->rank_tiles);
            k_rank_scan<<<(C + 127) / 128, 128, 0, c->stream>>>(c->rank_tiles, tiles, C);
            k_rank_assign<<<tiles, kRankTile, 4 * C, c->stream>>>(c->batch_of, n, C, c->rank_tiles, c->brank);
            c->launches += 3;
            GRB_CUDA(c, cudaGetLastError());
        }
        int nb = 0;
        GRB_CUDA(c, cudaMemcpy(&nb, c->ncolors, 4, cudaMemcpyDeviceToHost));
        k_plan_offsets<<<1, 1, 0, c->stream>>>(B, c->batch_off);
        if (n) k_plan_scatter<<<(n + 255) / 256, 256, 0, c->stream>>>(B, c->batch_off, c->ids);
        c->launches += n ? 2 : 1;
        GRB_CUDA(c, cudaGetLastError());
        GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
        c->h_batch_off.assign(nb + 1, 0);
        GRB_CUDA(c, cudaMemcpyAsync(c->h_batch_off.data(), c->batch_off, sizeof(int) * (nb + 1), cudaMemcpyDeviceToHost, c->stream));
        if (batch_of) GRB_CUDA(c, cudaMemcpyAsync(batch_of, c->batch_of, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        float ms = 0;
        GRB_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->batching_ms = ms;
        if ((rc = prof_collect(c))) return rc;
        c->plan_n = n;
        c->n_batches = nb;
        ++c->plan_version;
        if (n_batches) *n_batches = nb;
        return GRB_OK;
    }
    return fail(c, GRB_ELIMIT, "batch colours exceed the supported maximum");
}

int grb_refresh_cost(grb_ctx* c) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    return refresh_plain(c);
}

int grb_route_batch(grb_ctx* c, int32_t b, int32_t stamp) {
    if (!c || b < 0 || b >= c->n_batches) return c ? fail(c, GRB_EINVAL, "batch out of range") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    return route_plain(c, b, stamp);
}

int grb_commit_batch(grb_ctx* c, int32_t b, int32_t stamp, int32_t K) {
    if (!c || b < 0 || b >= c->n_batches || (K != 1 && K != -1)) return c ? fail(c, GRB_EINVAL, "bad commit arguments") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    return commit_plain(c, b, stamp, K);
}

int grb_lshape_stage(grb_ctx* c, int32_t mode, grb_stats* stats) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int stamp0 = c->stamp;
    GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int rc;
    c->tail_valid = 0;
    if ((rc = ensure_tail(c))) return rc;
    if (mode == GRB_MODE_PLAIN) rc = stage_plain(c, stamp0);
    else if (mode == GRB_MODE_GRAPH) rc = stage_graph(c, stamp0);
    else if (mode == GRB_MODE_PERSISTENT) rc = stage_persistent(c, stamp0);
    else return fail(c, GRB_EINVAL, "unknown mode");
    if (!rc && mode != GRB_MODE_PERSISTENT) rc = launch_tail(c);
    if (rc) return rc;
    GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    c->stamp = stamp0 + c->n_batches;
    if (c->tail_flags) { c->tail_valid = 1; c->tail_nets = c->n_nets; }
    rc = check_device_error(c);
    if (rc) return rc;
    float ms = 0;
    GRB_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->dag_ms = ms;
    if ((rc = prof_collect(c))) return rc;
    return stats ? grb_get_stats(c, stats) : GRB_OK;
}

int grb_set_flt_block_width(grb_ctx* c, int32_t width) {
    if (!c) return GRB_EINVAL;
    c->flt_block_width = width;
    return GRB_OK;
}

int grb_flt_stage(grb_ctx* c, int32_t remove_phase_one, int32_t mode, grb_stats* stats) {
    if (!c) return GRB_EINVAL;
    if (c->flt_n != c->n_nets || c->flt_n < 0) return fail(c, GRB_EINVAL, "no FLT DAGs uploaded for the current nets");
    GRB_CUDA(c, cudaSetDevice(c->device));
    std::vector<int> ids(c->plan_n);
    if (c->plan_n) {
        GRB_CUDA(c, cudaMemcpyAsync(ids.data(), c->ids, sizeof(int) * c->plan_n, cudaMemcpyDeviceToHost, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    for (int id : ids)
        if (c->h_flt_node_off[id + 1] == c->h_flt_node_off[id]) return fail(c, GRB_EINVAL, "plan net " + std::to_string(id) + " has no FLT DAG");
    if (c->flt_emap_plan != c->plan_version || c->flt_emap_flt != c->flt_version) {
        // Edge slots of the plan: each plan position's edges, in plan order.
        std::vector<int> eprefix(size_t(c->plan_n) + 1, 0);
        for (int k = 0; k < c->plan_n; ++k) {
            const long long e = eprefix[k] + (long long)c->h_flt_edge_off[ids[k] + 1] - c->h_flt_edge_off[ids[k]];
            if (e > INT_MAX / 81) return fail(c, GRB_EINVAL, "too many FLT edges in one plan");
            eprefix[k + 1] = int(e);
        }
        const long long slots = eprefix[c->plan_n];
        std::vector<int> emap(std::max(slots, 1ll));
        for (int k = 0; k < c->plan_n; ++k)
            std::fill(emap.begin() + eprefix[k], emap.begin() + eprefix[k + 1], k);
        if (c->flt_emap_cap < std::max<long long>(slots, c->plan_n + 1)) {
            if (c->flt_eprefix) cudaFree(c->flt_eprefix);
            if (c->flt_emap) cudaFree(c->flt_emap);
            c->flt_eprefix = c->flt_emap = nullptr;
            c->flt_emap_cap = 0;
            const long long cap = std::max<long long>(slots, c->plan_n + 1);
            if (cudaMalloc(&c->flt_eprefix, sizeof(int) * cap) != cudaSuccess ||
                cudaMalloc(&c->flt_emap, sizeof(int) * cap) != cudaSuccess) {
                cudaGetLastError();
                return fail(c, GRB_ENOMEM, "FLT edge map");
            }
            c->flt_emap_cap = cap;
        }
        GRB_CUDA(c, cudaMemcpyAsync(c->flt_eprefix, eprefix.data(), sizeof(int) * eprefix.size(), cudaMemcpyHostToDevice,
                                    c->stream));
        GRB_CUDA(c, cudaMemcpyAsync(c->flt_emap, emap.data(), sizeof(int) * slots, cudaMemcpyHostToDevice, c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->flt_emap_plan = c->plan_version;
        c->flt_emap_flt = c->flt_version;
    }
    c->F.eprefix = c->flt_eprefix;
    c->F.emap = c->flt_emap;
    const long long bkey[3] = {c->plan_version, c->flt_version, c->flt_block_width};
    if (!std::equal(bkey, bkey + 3, c->flt_border_key)) {
        // Each batch's positions with its wide nets first (a net's place inside
        // its batch changes nothing: the nets of a batch are independent).
        std::vector<int> border(std::max(c->plan_n, 1)), nwide(std::max(c->n_batches, 1), 0);
        for (int b = 0; b < c->n_batches; ++b) {
            int w = c->h_batch_off[b];
            for (int pass = 0; pass < 2; ++pass)
                for (int k = c->h_batch_off[b]; k < c->h_batch_off[b + 1]; ++k) {
                    const bool wide = c->flt_block_width >= 0 && c->h_flt_width[ids[k]] > c->flt_block_width;
                    if (wide == (pass == 0)) border[w++] = k;
                    if (wide && pass == 0) ++nwide[b];
                }
        }
        if (c->flt_border_cap < (long long)border.size() || c->flt_nwide_cap < (long long)nwide.size()) {
            if (c->flt_border) cudaFree(c->flt_border);
            if (c->flt_nwide) cudaFree(c->flt_nwide);
            c->flt_border = c->flt_nwide = nullptr;
            c->flt_border_cap = c->flt_nwide_cap = 0;
            if (cudaMalloc(&c->flt_border, sizeof(int) * border.size()) != cudaSuccess ||
                cudaMalloc(&c->flt_nwide, sizeof(int) * nwide.size()) != cudaSuccess) {
                cudaGetLastError();
                return fail(c, GRB_ENOMEM, "FLT net order");
            }
            c->flt_border_cap = (long long)border.size();
            c->flt_nwide_cap = (long long)nwide.size();
        }
        GRB_CUDA(c, cudaMemcpyAsync(c->flt_border, border.data(), sizeof(int) * border.size(), cudaMemcpyHostToDevice,
                                    c->stream));
        GRB_CUDA(c, cudaMemcpyAsync(c->flt_nwide, nwide.data(), sizeof(int) * nwide.size(), cudaMemcpyHostToDevice,
                                    c->stream));
        GRB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->h_flt_nwide = std::move(nwide);
        std::copy(bkey, bkey + 3, c->flt_border_key);
    }
    c->F.border = c->flt_border;
    c->F.nwide = c->flt_nwide;
    const int remove = remove_phase_one ? 1 : 0;
    const int stamp0 = c->stamp;
    GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int rc;
    if (mode == GRB_MODE_PLAIN) rc = flt_stage_plain(c, stamp0, remove);
    else if (mode == GRB_MODE_GRAPH) rc = flt_stage_graph(c, stamp0, remove);
    else if (mode == GRB_MODE_PERSISTENT) rc = flt_stage_persistent(c, stamp0, remove);
    else return fail(c, GRB_EINVAL, "unknown mode");
    if (rc) return rc;
    GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    c->stamp = stamp0 + flt_stamps(c, remove);
    rc = check_device_error(c);
    if (rc) return rc;
    float ms = 0;
    GRB_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->dag_ms = ms;
    if ((rc = prof_collect(c))) return rc;
    return stats ? grb_get_stats(c, stats) : GRB_OK;
}

int grb_softmin_forward(grb_ctx* c, int32_t dtype, double tau, const void* capacity, const void* unit_wire,
                        double unit_via, void* net_cost, double* total) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!(tau > 0) || !capacity || !unit_wire || !net_cost || !total) return fail(c, GRB_EINVAL, "bad soft-min arguments");
    if (dtype != GRB_F32 && dtype != GRB_F64) return fail(c, GRB_EINVAL, "dtype must be GRB_F32 or GRB_F64");
    GRB_CUDA(c, cudaSetDevice(c->device));
    int rc = soft_workspace(c);
    if (rc) return rc;
    if (dtype == GRB_F64)
        return soft_forward<double>(c, tau, capacity, unit_wire, unit_via, static_cast<double*>(net_cost), total);
    return soft_forward<float>(c, tau, capacity, unit_wire, unit_via, static_cast<float*>(net_cost), total);
}

int grb_softmin_backward(grb_ctx* c, int32_t dtype, double tau, const void* capacity, const void* unit_wire,
                         double unit_via, double grad_total, void* dcap, void* dunit_wire, double* dunit_via) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!(tau > 0) || !capacity || !unit_wire || !dcap || !dunit_wire || !dunit_via)
        return fail(c, GRB_EINVAL, "bad soft-min arguments");
    if (dtype != GRB_F32 && dtype != GRB_F64) return fail(c, GRB_EINVAL, "dtype must be GRB_F32 or GRB_F64");
    GRB_CUDA(c, cudaSetDevice(c->device));
    int rc = soft_workspace(c);
    if (rc) return rc;
    double duv = 0;
    if (dtype == GRB_F64)
        rc = soft_backward<double>(c, tau, capacity, unit_wire, unit_via, grad_total, static_cast<double*>(dcap),
                                   static_cast<double*>(dunit_wire), &duv);
    else
        rc = soft_backward<float>(c, tau, capacity, unit_wire, unit_via, grad_total, static_cast<float*>(dcap),
                                  static_cast<float*>(dunit_wire), &duv);
    if (rc) return rc;
    *dunit_via = duv;  // the adjoint already carries grad_total
    return GRB_OK;
}

int grb_zshape_stage(grb_ctx* c, int32_t mode, grb_stats* stats) {
    if (!c) return GRB_EINVAL;
    if (c->z_n != c->n_nets || c->z_n < 0) return fail(c, GRB_EINVAL, "no Z-shape trees uploaded for the current nets");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int stamp0 = c->stamp;
    GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int rc;
    if (mode == GRB_MODE_PLAIN) rc = z_stage_plain(c, stamp0);
    else if (mode == GRB_MODE_GRAPH) rc = z_stage_graph(c, stamp0);
    else if (mode == GRB_MODE_PERSISTENT) rc = z_stage_persistent(c, stamp0);
    else return fail(c, GRB_EINVAL, "unknown mode");
    if (rc) return rc;
    GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    c->stamp = stamp0 + c->n_batches;
    GRB_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0;
    GRB_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->dag_ms = ms;
    // As the reference (pipeline_ggr.hpp:136-138), a net without a finite
    // route or with a segment off the grid is reported after the whole stage
    // has run; its route record is left empty.
    rc = check_device_error(c);
    if (rc) return rc;
    if ((rc = prof_collect(c))) return rc;
    return stats ? grb_get_stats(c, stats) : GRB_OK;
}

int grb_read_routes2(grb_ctx* c, int32_t* routes2) {
    if (!c || !routes2) return GRB_EINVAL;
    if (c->flt_n < 0) return fail(c, GRB_EINVAL, "no FLT DAGs uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (c->route2_words)
        GRB_CUDA(c, cudaMemcpyAsync(routes2, c->F.routes2, sizeof(int) * c->route2_words, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_autotune(grb_ctx* c, int32_t what, int32_t* per_cta, int32_t* per_grab) {
    if (!c) return GRB_EINVAL;
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    if (!c->n_batches) return fail(c, GRB_EINVAL, "no plan to tune on");
    GRB_CUDA(c, cudaSetDevice(c->device));
    int rc = ensure_buckets(c);
    if (rc) return rc;
    const bool prof = c->profiling;
    c->profiling = false;
    if (what & 1) {
        // Per-batch DP form: coordinate descent over the buckets -- for each
        // bucket in turn, time the whole per-batch launch of the three largest
        // batches with each nets-per-CTA choice (DP only, on refreshed tables).
        if ((rc = refresh_plain(c))) { c->profiling = prof; return rc; }
        std::vector<int> order(c->n_batches);
        for (int b = 0; b < c->n_batches; ++b) order[b] = b;
        std::sort(order.begin(), order.end(), [&](int a, int b) {
            return c->h_batch_off[a + 1] - c->h_batch_off[a] > c->h_batch_off[b + 1] - c->h_batch_off[b];
        });
        const int samples = std::min<int>(3, order.size());
        for (int bk = 0; bk < kDpBuckets; ++bk) {
            float best = 1e30f;
            int choice = c->tune.per_cta[bk];
            for (int per : {1, 2, 4, 8}) {
                c->tune.per_cta[bk] = per;
                float ms = 1e30f;
                for (int rep = 0; rep < 3 && !rc; ++rep) {
                    GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
                    for (int q = 0; q < samples && !rc; ++q) rc = launch_buckets(c, order[q], c->stamp + 1, -1);
                    GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
                    GRB_CUDA(c, cudaEventSynchronize(c->ev1));
                    float t = 0;
                    GRB_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
                    ms = std::min(ms, t);
                }
                if (rc) { c->profiling = prof; return rc; }
                if (ms < best) { best = ms; choice = per; }
            }
            c->tune.per_cta[bk] = choice;
        }
        if ((rc = check_device_error(c))) { c->profiling = prof; return rc; }
    }
    if (what & 2) {
        // Persistent form: whole-stage runs from a reset state for each
        // candidate set of nets per grab (small buckets take more per grab).
        // per_grab[0] >= 32: nets of one or two nodes one per lane, that many
        // per grab.
        constexpr int kCands = 6;
        const int cands[kCands][kDpBuckets] = {{1, 1, 1, 1}, {2, 1, 1, 1}, {4, 2, 1, 1}, {8, 4, 2, 1},
                                               {32, 2, 1, 1}, {64, 4, 2, 1}};
        float best = 1e30f;
        int pick = 0;
        for (int k = 0; k < kCands; ++k) {
            for (int q = 0; q < kDpBuckets; ++q) c->tune.per_grab[q] = cands[k][q];
            if ((rc = grb_reset(c))) { c->profiling = prof; return rc; }
            GRB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
            if ((rc = stage_persistent(c, 0))) { c->profiling = prof; return rc; }
            GRB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
            GRB_CUDA(c, cudaEventSynchronize(c->ev1));
            float t = 0;
            GRB_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
            if ((rc = check_device_error(c))) { c->profiling = prof; return rc; }
            if (t < best) { best = t; pick = k; }
        }
        for (int q = 0; q < kDpBuckets; ++q) c->tune.per_grab[q] = cands[pick][q];
    }
    c->profiling = prof;
    c->graph_version = -1;  // a captured per-batch sequence bakes in the launch shapes
    if ((rc = grb_reset(c))) return rc;
    for (int q = 0; q < kDpBuckets; ++q) {
        if (per_cta) per_cta[q] = c->tune.per_cta[q];
        if (per_grab) per_grab[q] = c->tune.per_grab[q];
    }
    return GRB_OK;
}

static int ripup_classify(grb_ctx* c, int32_t threshold, const uint8_t* phase2, uint8_t* is_of);

int grb_ripup_classify(grb_ctx* c, int32_t threshold, uint8_t* is_of) {
    return ripup_classify(c, threshold, nullptr, is_of);
}

int grb_ripup_classify_phase2(grb_ctx* c, int32_t threshold, const uint8_t* phase2, uint8_t* is_of) {
    if (!c || !phase2) return c ? fail(c, GRB_EINVAL, "null flags") : GRB_EINVAL;
    for (int id = 0; id < c->n_nets; ++id)
        if (phase2[id] && (c->flt_n != c->n_nets || c->h_route2_off[id + 1] == c->h_route2_off[id]))
            return fail(c, GRB_EINVAL, "net " + std::to_string(id) + " has no phase-two routes");
    return ripup_classify(c, threshold, phase2, is_of);
}

static int ripup_classify(grb_ctx* c, int32_t threshold, const uint8_t* phase2, uint8_t* is_of) {
    if (!c || !is_of) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    int* of_sum = nullptr;
    unsigned char* flags = nullptr;
    unsigned char* d_phase2 = nullptr;
    if (cudaMalloc(&of_sum, sizeof(int) * size_t(c->T.cells)) || cudaMalloc(&flags, std::max(c->n_nets, 1)) ||
        (phase2 && cudaMalloc(&d_phase2, std::max(c->n_nets, 1)))) {
        cudaGetLastError();
        if (of_sum) cudaFree(of_sum);
        if (flags) cudaFree(flags);
        return fail(c, GRB_ENOMEM, "rip-up buffers");
    }
    if (phase2 && c->n_nets)
        GRB_CUDA(c, cudaMemcpyAsync(d_phase2, phase2, size_t(c->n_nets), cudaMemcpyHostToDevice, c->stream));
    int tracks = 0;
    for (int l = 0; l < c->T.L; ++l) tracks += (((l & 1) ^ c->T.DIR) ? c->T.X : c->T.Y);
    k_mark_overflow<<<(c->T.cells + 255) / 256, 256, 0, c->stream>>>(c->T, threshold, of_sum);
    k_int_prefix<<<(tracks + 127) / 128, 128, 0, c->stream>>>(c->T, of_sum);
    Plan P = make_plan(c);
    if (c->n_nets && phase2)
        k_overflow_nets2<<<(c->n_nets + 255) / 256, 256, 0, c->stream>>>(c->T, P, make_plan2(c), c->n_nets, of_sum,
                                                                           d_phase2, flags);
    else if (c->n_nets)
        k_overflow_nets<<<(c->n_nets + 255) / 256, 256, 0, c->stream>>>(c->T, P, c->n_nets, of_sum, flags);
    c->launches += 3;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(is_of, flags, c->n_nets, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(of_sum);
    cudaFree(flags);
    if (d_phase2) cudaFree(d_phase2);
    if (e != cudaSuccess) return cuda_fail(c, e, "rip-up classification");
    return GRB_OK;
}

// Device address of g_noalloc_scratch on the current device.  Host code only
// holds a host-side stand-in for the array's name, so the address is looked up
// once per device, with that device current, and cached until the process
// exits (a device reset by the host application invalidates it).
static int noalloc_scratch(grb_ctx* c, int** out) {
    static std::mutex lock;
    static std::vector<int*> cache;
    std::lock_guard<std::mutex> guard(lock);
    if (c->device >= int(cache.size())) cache.resize(c->device + 1, nullptr);
    if (!cache[c->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        cache[c->device] = static_cast<int*>(p);
    }
    *out = cache[c->device];
    return GRB_OK;
}

int grb_ripup_classify_noalloc(grb_ctx* c, int32_t threshold, uint8_t* is_of) {
    if (!c || !is_of) return c ? fail(c, GRB_EINVAL, "is_of must not be NULL") : GRB_EINVAL;
    if (c->T.cells > kNoAllocCells)
        return fail(c, GRB_ELIMIT, "grid has " + std::to_string(c->T.cells) + " cells; the allocation-free "
                    "classification supports at most " + std::to_string(kNoAllocCells));
    if (c->n_nets > kNoAllocNets)
        return fail(c, GRB_ELIMIT, "design has " + std::to_string(c->n_nets) + " nets; the allocation-free "
                    "classification supports at most " + std::to_string(kNoAllocNets));
    if (!c->node_off) return fail(c, GRB_EINVAL, "no nets uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    int* scratch = nullptr;
    const int rc = noalloc_scratch(c, &scratch);
    if (rc) return rc;
    // Every scratch word used below is written before it is read (one overflow
    // mark per cell, one flag per net), so nothing has to be cleared first.
    int* of_sum = scratch;
    unsigned char* flags = reinterpret_cast<unsigned char*>(scratch + kNoAllocCells);
    int tracks = 0;
    for (int l = 0; l < c->T.L; ++l) tracks += (((l & 1) ^ c->T.DIR) ? c->T.X : c->T.Y);
    k_mark_overflow<<<(c->T.cells + 255) / 256, 256, 0, c->stream>>>(c->T, threshold, of_sum);
    k_int_prefix<<<(tracks + 127) / 128, 128, 0, c->stream>>>(c->T, of_sum);
    Plan P = make_plan(c);
    if (c->n_nets) k_overflow_nets<<<(c->n_nets + 255) / 256, 256, 0, c->stream>>>(c->T, P, c->n_nets, of_sum, flags);
    c->launches += c->n_nets ? 3 : 2;
    GRB_CUDA(c, cudaGetLastError());
    if (c->n_nets) GRB_CUDA(c, cudaMemcpyAsync(is_of, flags, c->n_nets, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_set_stage_tail(grb_ctx* c, int32_t flags, int32_t threshold) {
    if (!c) return GRB_EINVAL;
    if (flags & ~(kTailRipup | kTailView)) return fail(c, GRB_EINVAL, "unknown stage tail flags");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const size_t cells = c->T.cells, xy = c->T.XY;
    if ((flags & kTailRipup) && !c->tail_of_sum && cudaMalloc(&c->tail_of_sum, 4 * cells) != cudaSuccess) {
        cudaGetLastError();
        c->tail_of_sum = nullptr;
        return fail(c, GRB_ENOMEM, "rip-up marks");
    }
    if ((flags & kTailView) && !c->tail_cong) {
        if (cudaMalloc(&c->tail_cong, xy) || cudaMalloc(&c->tail_xsum, 4 * xy) || cudaMalloc(&c->tail_ysum, 4 * xy)) {
            cudaGetLastError();
            for (void* p : {(void*)c->tail_cong, (void*)c->tail_xsum, (void*)c->tail_ysum}) if (p) cudaFree(p);
            c->tail_cong = nullptr; c->tail_xsum = c->tail_ysum = nullptr;
            return fail(c, GRB_ENOMEM, "congestion view buffers");
        }
    }
    c->tail_flags = flags;
    c->tail_threshold = threshold;
    c->tail_valid = 0;
    return ensure_tail(c);
}

int grb_read_stage_tail(grb_ctx* c, uint8_t* is_of, uint8_t* congestion, float* xsum, float* ysum) {
    if (!c) return GRB_EINVAL;
    if (!c->tail_valid) return fail(c, GRB_EINVAL, "no L-shape stage has run with a stage tail since it was set");
    if (is_of && !(c->tail_flags & kTailRipup)) return fail(c, GRB_EINVAL, "the stage tail has no rip-up classification");
    if ((congestion || xsum || ysum) && !(c->tail_flags & kTailView))
        return fail(c, GRB_EINVAL, "the stage tail has no congestion view");
    GRB_CUDA(c, cudaSetDevice(c->device));
    const size_t xy = c->T.XY;
    if (is_of && c->tail_nets) GRB_CUDA(c, cudaMemcpyAsync(is_of, c->tail_is_of, c->tail_nets, cudaMemcpyDeviceToHost, c->stream));
    if (congestion) GRB_CUDA(c, cudaMemcpyAsync(congestion, c->tail_cong, xy, cudaMemcpyDeviceToHost, c->stream));
    if (xsum) GRB_CUDA(c, cudaMemcpyAsync(xsum, c->tail_xsum, 4 * xy, cudaMemcpyDeviceToHost, c->stream));
    if (ysum) GRB_CUDA(c, cudaMemcpyAsync(ysum, c->tail_ysum, 4 * xy, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_cost_exp(int32_t device, const float* x, int32_t n, float* y) {
    if (n < 0 || (n > 0 && (!x || !y))) return GRB_EINVAL;
    if (n == 0) return GRB_OK;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return GRB_ECUDA; }
    float* d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * 2 * size_t(n)) != cudaSuccess) { cudaGetLastError(); return GRB_ENOMEM; }
    cudaError_t e = cudaMemcpy(d, x, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_cost_exp<<<std::min((n + 255) / 256, 4096), 256>>>(d, n, d + n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + n, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { cudaGetLastError(); return GRB_ECUDA; }
    return GRB_OK;
}

int grb_congestion_view(grb_ctx* c, uint8_t* congestion, float* xsum, float* ysum) {
    if (!c || !congestion || !xsum || !ysum) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int X = c->T.X, Y = c->T.Y, XY = c->T.XY;
    unsigned char* d_c = nullptr;
    float *d_x = nullptr, *d_y = nullptr;
    if (cudaMalloc(&d_c, XY) || cudaMalloc(&d_x, 4 * size_t(XY)) || cudaMalloc(&d_y, 4 * size_t(XY))) {
        cudaGetLastError();
        for (void* p : {(void*)d_c, (void*)d_x, (void*)d_y}) if (p) cudaFree(p);
        return fail(c, GRB_ENOMEM, "congestion buffers");
    }
    k_congestion<<<(XY + 255) / 256, 256, 0, c->stream>>>(c->T, d_c, d_x, d_y);
    k_float_line_prefix<<<(X + 127) / 128, 128, 0, c->stream>>>(d_y, X, Y, Y, 1);   // per x, along y
    k_float_line_prefix<<<(Y + 127) / 128, 128, 0, c->stream>>>(d_x, Y, X, 1, Y);   // per y, along x
    c->launches += 3;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(congestion, d_c, XY, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(xsum, d_x, 4 * size_t(XY), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ysum, d_y, 4 * size_t(XY), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_c); cudaFree(d_x); cudaFree(d_y);
    if (e != cudaSuccess) return cuda_fail(c, e, "congestion view");
    return GRB_OK;
}

int grb_read_tables(grb_ctx* c, float* wcost, float* vcost, double* presum, int32_t* demand_half, int32_t* timestamp) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const size_t cells = c->T.cells;
    if (wcost) GRB_CUDA(c, cudaMemcpyAsync(wcost, c->T.wcost, 4 * cells, cudaMemcpyDeviceToHost, c->stream));
    if (vcost) GRB_CUDA(c, cudaMemcpyAsync(vcost, c->T.vcost, 4 * cells, cudaMemcpyDeviceToHost, c->stream));
    if (presum) GRB_CUDA(c, cudaMemcpyAsync(presum, c->T.presum, 8 * cells, cudaMemcpyDeviceToHost, c->stream));
    if (demand_half) GRB_CUDA(c, cudaMemcpyAsync(demand_half, c->T.demand, 4 * cells, cudaMemcpyDeviceToHost, c->stream));
    if (timestamp) GRB_CUDA(c, cudaMemcpyAsync(timestamp, c->T.ts, 4 * cells, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int grb_read_routes(grb_ctx* c, int32_t* routes) {
    if (!c || !routes) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (c->route_words) GRB_CUDA(c, cudaMemcpyAsync(routes, c->routes, sizeof(int) * c->route_words, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

// Host side of the used-word transfers: device positions for n nets and a
// packed buffer of `words` (grown as needed), and the host route offsets.
static int used_buffers(grb_ctx* c, long long words) {
    const int n = c->n_nets;
    if (c->used_n_cap < n) {
        free_all(c->used_bufs);
        c->used_words_cap = 0;
        c->used_pack = nullptr;
        const int tiles = (n + kScanTile - 1) / kScanTile;
        if (dalloc(c, &c->used_pos, size_t(n) + 1, c->used_bufs) || dalloc(c, &c->used_sums, size_t(tiles) + 1, c->used_bufs)) {
            free_all(c->used_bufs);
            c->used_n_cap = -1;
            return fail(c, GRB_ENOMEM, "route transfer positions");
        }
        c->used_n_cap = n;
    }
    if (words > c->used_words_cap) {
        if (c->used_pack) {
            cudaFree(c->used_pack);
            c->used_bufs.erase(std::find(c->used_bufs.begin(), c->used_bufs.end(), (void*)c->used_pack));
            c->used_pack = nullptr;
            c->used_words_cap = 0;
        }
        if (dalloc(c, &c->used_pack, size_t(std::max(words, 1ll)), c->used_bufs)) return fail(c, GRB_ENOMEM, "route transfer buffer");
        c->used_words_cap = words;
    }
    return GRB_OK;
}

// Copy each net's words in use between `host` (at the route offsets) and
// `packed` (at the positions), on `threads` host threads.
static void used_scatter(int n, const long long* route_off, const long long* pos, int* host, int* packed,
                         bool to_host) {
    const int threads = int(std::min<long long>(8, std::max(1, n / 4096)));
    auto part = [&](int t) {
        const int lo = int((long long)n * t / threads), hi = int((long long)n * (t + 1) / threads);
        for (int i = lo; i < hi; ++i) {
            const size_t m = size_t(pos[i + 1] - pos[i]);
            if (to_host) std::memcpy(host + route_off[i], packed + pos[i], m * sizeof(int));
            else std::memcpy(packed + pos[i], host + route_off[i], m * sizeof(int));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(part, t);
    part(0);
    for (auto& th : pool) th.join();
}

int grb_read_routes_used(grb_ctx* c, int32_t* routes) {
    if (!c || !routes) return c ? fail(c, GRB_EINVAL, "null routes") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n_nets;
    if (n <= 0) return GRB_OK;
    int rc = used_buffers(c, 0);
    if (rc) return rc;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    k_route_used<<<(n + 255) / 256, 256, 0, c->stream>>>(c->routes, c->route_off, n, c->used_pos);
    k_scan_tiles<<<tiles, 256, 0, c->stream>>>(c->used_pos, n, c->used_sums);
    k_scan_sums<<<1, 1024, 0, c->stream>>>(c->used_sums, tiles);
    k_scan_add<<<n / 256 + 1, 256, 0, c->stream>>>(c->used_pos, n, c->used_sums, tiles);
    c->launches += 4;
    GRB_CUDA(c, cudaGetLastError());
    std::vector<long long> pos(size_t(n) + 1), off(size_t(n) + 1);
    GRB_CUDA(c, cudaMemcpyAsync(pos.data(), c->used_pos, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(off.data(), c->route_off, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    const long long words = pos[n];
    if ((rc = used_buffers(c, words))) return rc;
    k_route_move<<<std::max(1, std::min((n + 7) / 8, c->sms * 16)), 256, 0, c->stream>>>(c->route_off, c->used_pos, n,
                                                                                        c->routes, c->used_pack, 1);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    std::vector<int> packed(size_t(std::max(words, 1ll)));
    GRB_CUDA(c, cudaMemcpyAsync(packed.data(), c->used_pack, sizeof(int) * words, cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    used_scatter(n, off.data(), pos.data(), routes, packed.data(), true);
    return GRB_OK;
}

int grb_write_routes_used(grb_ctx* c, const int32_t* routes) {
    if (!c || !routes) return c ? fail(c, GRB_EINVAL, "null routes") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n_nets;
    if (n <= 0) return GRB_OK;
    std::vector<long long> pos(size_t(n) + 1), off(size_t(n) + 1);
    GRB_CUDA(c, cudaMemcpyAsync(off.data(), c->route_off, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    pos[0] = 0;
    for (int i = 0; i < n; ++i) {
        const long long cap = off[i + 1] - off[i];
        pos[i + 1] = pos[i] + (cap > 0 ? std::max(1ll, std::min<long long>(routes[off[i]], cap)) : 0);
    }
    const long long words = pos[n];
    int rc = used_buffers(c, words);
    if (rc) return rc;
    std::vector<int> packed(size_t(std::max(words, 1ll)));
    used_scatter(n, off.data(), pos.data(), const_cast<int32_t*>(routes), packed.data(), false);
    GRB_CUDA(c, cudaMemcpyAsync(c->used_pack, packed.data(), sizeof(int) * words, cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(c->used_pos, pos.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, c->stream));
    k_route_move<<<std::max(1, std::min((n + 7) / 8, c->sms * 16)), 256, 0, c->stream>>>(c->route_off, c->used_pos, n,
                                                                                        c->routes, c->used_pack, 0);
    c->launches += 1;
    GRB_CUDA(c, cudaGetLastError());
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_write_routes(grb_ctx* c, const int32_t* routes) {
    if (!c || !routes) return c ? fail(c, GRB_EINVAL, "null routes") : GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (c->route_words)
        GRB_CUDA(c, cudaMemcpyAsync(c->routes, routes, sizeof(int) * c->route_words, cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_write_routes2(grb_ctx* c, const int32_t* routes2) {
    if (!c || !routes2) return c ? fail(c, GRB_EINVAL, "null routes") : GRB_EINVAL;
    if (c->flt_n != c->n_nets || c->flt_n < 0) return fail(c, GRB_EINVAL, "no phase-two route storage uploaded");
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (c->route2_words)
        GRB_CUDA(c, cudaMemcpyAsync(c->F.routes2, routes2, sizeof(int) * c->route2_words, cudaMemcpyHostToDevice,
                                    c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_get_stats(grb_ctx* c, grb_stats* s) {
    if (!c || !s) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    unsigned long long v = 0;
    GRB_CUDA(c, cudaMemcpyAsync(&s->total_wirelength, c->T.wirelength, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(&v, c->T.vias, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    s->total_via_count = static_cast<int64_t>(v);
    s->n_batches = c->n_batches;
    s->stamp = c->stamp;
    s->batching_ms = c->batching_ms;
    s->dag_ms = c->dag_ms;
    return GRB_OK;
}

int grb_set_stats(grb_ctx* c, double wirelength, int64_t vias) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    const unsigned long long v = static_cast<unsigned long long>(vias);
    GRB_CUDA(c, cudaMemcpyAsync(c->T.wirelength, &wirelength, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaMemcpyAsync(c->T.vias, &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return GRB_OK;
}

int grb_sync(grb_ctx* c) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    GRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int64_t grb_kernel_launches(grb_ctx* c) { return c ? c->launches : 0; }

int grb_set_wait_limit(grb_ctx* c, double seconds) {
    if (!c) return GRB_EINVAL;
    if (!(seconds > 0) || seconds > 3600) return fail(c, GRB_EINVAL, "wait limit must be in (0, 3600] seconds");
    c->wait_ns = static_cast<unsigned long long>(seconds * 1e9);
    if (c->wait_ns == 0) c->wait_ns = 1;
    return GRB_OK;
}

int grb_set_profiling(grb_ctx* c, int32_t on) {
    if (!c) return GRB_EINVAL;
    GRB_CUDA(c, cudaSetDevice(c->device));
    if (on && !c->d_phase) {
        if (cudaMalloc(&c->d_phase, kPhaseSlots * sizeof(unsigned long long)) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GRB_ENOMEM, "profiling buffer");
        }
        GRB_CUDA(c, cudaMemset(c->d_phase, 0, kPhaseSlots * sizeof(unsigned long long)));
    }
    c->profiling = on != 0;
    return GRB_OK;
}

int grb_phase_times(grb_ctx* c, double* ms, int32_t n, int32_t reset) {
    if (!c || !ms || n < 0) return GRB_EINVAL;
    for (int k = 0; k < n && k < kPhaseSlots; ++k) ms[k] = c->phase_ms[k];
    if (reset) for (double& v : c->phase_ms) v = 0;
    return GRB_OK;
}

}  // extern "C"
