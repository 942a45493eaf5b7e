// batching.cuh -- exact greedy first-fit net batching on the GPU.
//
// Semantics of the reference's CPU batching (generate_batches_cpu.hpp:7-73):
// nets are taken in the given order; a net joins the first batch that holds
// fewer than `limit` nets and none of whose marked cells contains one of the
// net's query points; it then marks its RSMT h-segments (step sparsity*Y),
// v-segments (step sparsity) and, at every point, the cell itself, its x
// neighbours and the cell below in y (not above, reference :38).
//
// B200 algorithm (replaces the RT-core/OptiX and CPU paths, which produce the
// same lists):
//   * cellmask[cell] holds one bit per batch ("colour") already marking the cell;
//   * nets are processed in chunks of 512 in order; per chunk:
//       1. every net rasters its marks into a chunk-local bitmask per cell
//          (bit = its position in the chunk) and ORs cellmask over its points
//          -> forbidden colours from earlier chunks;
//       2. every net ORs the chunk-local masks over its points, keeping bits of
//          earlier chunk nets -> exact intra-chunk predecessors;
//       3. one CTA solves first-fit inside the chunk by Jacobi iteration over
//          the predecessor DAG (converges to the unique sequential solution),
//          then applies batch capacities in order;
//       4. every net ORs its colour into cellmask over its marks and clears the
//          chunk-local masks.
//   The chunks run inside one cooperative kernel with bounded grid barriers
//   (persistent form) or as one launch per phase (plain form).  The chunk-local
//   masks are double-buffered by chunk parity, so the persistent form rasters
//   chunk k+1 on every other CTA while one CTA solves chunk k, and reads the
//   forbidden colours (step 1's second half) together with the predecessors
//   after chunk k-1 is published.
#pragma once
#include "common.cuh"

namespace grb {

constexpr int kChunk = 512;     // nets per chunk (== threads of the solve CTA)
constexpr int kChunkWords = kChunk / 32;

struct BatchState {
    int X, Y, n, limit, sparsity, W;   // W: colour words per cell
    const int* order;
    const int* point_off; const int* points;
    const int* hseg_off; const int* hsegs;
    const int* vseg_off; const int* vsegs;
    unsigned* cellmask;    // [X*Y][W]
    unsigned* localmask;   // [X*Y][kChunkWords], chunks of even index
    unsigned* localmask2;  // [X*Y][kChunkWords], chunks of odd index
    unsigned* fmask;       // [W][kChunk] (word-major: the solve copies it as is)
    unsigned* pred;        // [kChunkWords][kChunk]
    unsigned* fullmask;    // [W]
    int* count;            // [32*W]
    int* n_colors;         // [1]
    int* batch_of;         // [n] colour per order position
    int* rank;             // [n] position inside its batch
    int* error;
    int* error_info;
};

__device__ __forceinline__ void batch_error(const BatchState& B, int code, int info) {
    if (atomicCAS(B.error, 0, code) == 0) *B.error_info = info;
}

// Cells of the segments [s0, s1) of `segs` with step `step`; threads t of n
// split each segment's cells.  Every warp of the group fetches 32 segment
// endpoints per memory round trip and broadcasts them by shuffle, so a net
// with many short segments does not wait one load latency per segment.
// All 32 lanes of each warp of the group must call this.
template <class F>
__device__ __forceinline__ void for_each_segment_cell(const int* segs, int s0, int s1, int step, int t, int n, F f) {
    const int lane = t & 31;
    for (int base = s0; base < s1; base += 32) {
        int a = 0, b = -1;
        if (base + lane < s1) { a = segs[2 * (base + lane)]; b = segs[2 * (base + lane) + 1]; }
        const int m = min(32, s1 - base);
        for (int q = 0; q < m; ++q) {
            const int aq = __shfl_sync(0xffffffffu, a, q), bq = __shfl_sync(0xffffffffu, b, q);
            if (bq < aq) continue;
            const int cnt = (bq - aq) / step + 1;
            for (int k = t; k < cnt; k += n) f(aq + k * step);
        }
    }
}

// Visit every cell net `id` marks (duplicates allowed); threads t of n split
// the work.
template <class F>
__device__ __forceinline__ void for_each_mark(const BatchState& B, int id, int t, int n, F f) {
    for_each_segment_cell(B.hsegs, B.hseg_off[id], B.hseg_off[id + 1], B.sparsity * B.Y, t, n, f);
    for_each_segment_cell(B.vsegs, B.vseg_off[id], B.vseg_off[id + 1], B.sparsity, t, n, f);
    const int p0 = B.point_off[id], np = B.point_off[id + 1] - p0;
    for (int k = t; k < 4 * np; k += n) {
        const int p = B.points[p0 + k / 4], x = p / B.Y, y = p - x * B.Y;
        const int which = k & 3;
        int cx = x, cy = y;
        if (which == 0) cx = x - 1;
        else if (which == 1) cy = y - 1;
        else if (which == 3) cx = x + 1;
        if (cx >= 0 && cx < B.X && cy >= 0) f(cx * B.Y + cy);
    }
}

// A group of threads that works on one net: a whole CTA, or half of one
// synchronised with a named barrier.
struct NetGroup {
    int t, n, bar;  // thread rank, group size, named barrier id (0: the CTA)
    __device__ __forceinline__ void sync() const {
        if (bar == 0) __syncthreads();
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(n) : "memory");
    }
};

// Chunk-local mask buffer of the chunk starting at order position s.
__device__ __forceinline__ unsigned* chunk_mask(const BatchState& B, int s) {
    return ((s / kChunk) & 1) ? B.localmask2 : B.localmask;
}

// The per-net steps run one net per group (its threads share the net's marks
// and points).
// Step 1a: chunk-local raster.
__device__ __forceinline__ void batch_raster(const BatchState& B, int s, int jj, const NetGroup& G) {
    const int id = B.order[s + jj];
    const unsigned bit = 1u << (jj & 31);
    const int word = jj >> 5;
    unsigned* lm = chunk_mask(B, s);
    for_each_mark(B, id, G.t, G.n, [&](int q) { red_or(lm + size_t(q) * kChunkWords + word, bit); });
}

// Step 1b + 2: forbidden colours from earlier (published) chunks and the
// predecessors inside the chunk, both ORed over the net's query points.
// `acc` is group shared memory of W + kChunkWords words.
__device__ __forceinline__ void batch_forbid_preds(const BatchState& B, int s, int jj, unsigned* acc, const NetGroup& G) {
    const int id = B.order[s + jj];
    const int t = G.t, n = G.n;
    const int W = B.W;
    const int words = (jj >> 5) + 1;  // only bits of earlier chunk nets matter
    const unsigned* lm = chunk_mask(B, s);
    for (int w = t; w < W + kChunkWords; w += n) acc[w] = 0u;
    G.sync();
    const int p0 = B.point_off[id], np = B.point_off[id + 1] - p0;
    for (int k = t; k < np * W; k += n) {
        const int w = k % W;
        const unsigned v = B.cellmask[size_t(B.points[p0 + k / W]) * W + w];
        if (v) atomicOr(acc + w, v);
    }
    for (int k = t; k < np * words; k += n) {
        const int w = k % words;
        const unsigned v = lm[size_t(B.points[p0 + k / words]) * kChunkWords + w];
        if (v) atomicOr(acc + W + w, v);
    }
    G.sync();
    for (int w = t; w < W; w += n) B.fmask[size_t(w) * kChunk + jj] = acc[w];
    for (int w = t; w < kChunkWords; w += n) {
        unsigned v = w < words ? acc[W + w] : 0u;
        if (w == (jj >> 5)) v &= (1u << (jj & 31)) - 1u;
        B.pred[w * kChunk + jj] = v;
    }
    G.sync();
}

// Phase 4: publish the net's colour over its marks and clear its chunk-local
// word (every net of the chunk clears the word holding its own bit, so all
// words touched by the chunk end up zero).
__device__ __forceinline__ void batch_phase4(const BatchState& B, int s, int jj, const NetGroup& G) {
    const int id = B.order[s + jj];
    const int c = B.batch_of[s + jj];
    const unsigned bit = 1u << (c & 31);
    const int word = c >> 5, lword = jj >> 5;
    unsigned* lm = chunk_mask(B, s);
    for_each_mark(B, id, G.t, G.n, [&](int q) {
        red_or(B.cellmask + size_t(q) * B.W + word, bit);
        lm[size_t(q) * kChunkWords + lword] = 0u;
    });
}

// Phase 3 (one CTA of kChunk threads): first-fit inside the chunk.
// smem (word-major so a warp reads 32 consecutive words): F[W][kChunk],
// P[kChunkWords][kChunk], col[kChunk], cnt[32W], run[32W], full[W].
__device__ void batch_phase3(const BatchState& B, int s, unsigned* smem) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m = min(kChunk, B.n - s);
    const int W = B.W, C = 32 * W;
    unsigned* F = smem;
    unsigned* P = F + kChunk * W;
    int* col = reinterpret_cast<int*>(P + kChunk * kChunkWords);
    int* cnt = col + kChunk;
    int* run = cnt + C;
    unsigned* full = reinterpret_cast<unsigned*>(run + C);
    __shared__ int first_bad, overflow;
    // Both tables are word-major in global memory already: 16-byte copies.
    {
        const uint4* f4 = reinterpret_cast<const uint4*>(B.fmask);
        const uint4* p4 = reinterpret_cast<const uint4*>(B.pred);
        uint4* F4 = reinterpret_cast<uint4*>(F);
        uint4* P4 = reinterpret_cast<uint4*>(P);
        const int nf = W * kChunk / 4, np = kChunkWords * kChunk / 4;
        for (int k = tid; k < nf + np; k += blockDim.x) {
            if (k < nf) F4[k] = f4[k];
            else P4[k - nf] = p4[k - nf];
        }
    }
    for (int k = tid; k < C; k += blockDim.x) cnt[k] = B.count[k];
    for (int k = tid; k < W; k += blockDim.x) full[k] = B.fullmask[k];
    if (tid < kChunk) col[tid] = -1;
    if (tid == 0) overflow = 0;
    __syncthreads();
    int fixed = 0;  // nets below `fixed` are final
    int rank = 0;
    while (true) {
        // Jacobi sweeps until the colouring is a fixed point: a net's colour is
        // the first one neither forbidden by earlier chunks, nor full, nor held
        // by one of its predecessors in the chunk.
        while (true) {
            int mine = tid < m ? col[tid] : -1;
            if (tid < m && tid >= fixed) {
                int c = 0;
                while (true) {
                    int w = c >> 5;
                    if (w >= W) { c = C; break; }
                    unsigned used = F[w * kChunk + tid] | full[w] | ((1u << (c & 31)) - 1u);
                    while (used == 0xffffffffu) {
                        if (++w >= W) break;
                        used = F[w * kChunk + tid] | full[w];
                    }
                    if (w >= W) { c = C; break; }
                    c = w * 32 + __ffs(~used) - 1;
                    bool hit = false;
                    for (int pw = 0; pw <= (tid >> 5) && !hit; ++pw) {
                        unsigned bits = P[pw * kChunk + tid];
                        while (bits) {
                            const int i = pw * 32 + __ffs(bits) - 1;
                            bits &= bits - 1;
                            if (col[i] == c) { hit = true; break; }
                        }
                    }
                    if (!hit) break;
                    ++c;
                }
                if (c >= C) { overflow = 1; c = C - 1; }
                mine = c;
            }
            __syncthreads();
            const bool changed = tid < m && col[tid] != mine;
            if (tid < m) col[tid] = mine;
            if (!__syncthreads_or(changed)) break;
        }
        if (overflow) break;
        // Position of every net inside its batch, in chunk order: warps in turn
        // add their per-colour group sizes to a running count.
        for (int k = tid; k < C; k += blockDim.x) run[k] = cnt[k];
        if (tid == 0) first_bad = m;
        __syncthreads();
        const int c = tid < m ? col[tid] : -1 - lane;  // distinct dummies for idle lanes
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int within = __popc(peers & ((1u << lane) - 1u));
        for (int w = 0; w < (m + 31) / 32; ++w) {
            if (warp == w && tid < m) {
                rank = run[c] + within;
                if (lane == __ffs(peers) - 1) run[c] += __popc(peers);
                if (rank >= B.limit) atomicMin(&first_bad, tid);
            }
            __syncthreads();
        }
        const int bad = first_bad;
        if (bad >= m) {
            if (tid < m) {
                B.batch_of[s + tid] = col[tid];
                B.rank[s + tid] = rank;
            }
            for (int k = tid; k < C; k += blockDim.x) cnt[k] = run[k];
            __syncthreads();
            break;
        }
        // Net `bad` finds its colour full; so does every later net.
        const int full_colour = col[bad];
        __syncthreads();
        if (tid == 0) full[full_colour >> 5] |= 1u << (full_colour & 31);
        fixed = bad;
        __syncthreads();
    }
    if (overflow) {
        if (tid == 0) batch_error(B, kELimit, s);
        return;
    }
    int top = 0;
    if (tid < m) top = col[tid] + 1;
    for (int k = tid; k < C; k += blockDim.x) B.count[k] = cnt[k];
    for (int k = tid; k < W; k += blockDim.x) B.fullmask[k] = full[k];
    if (top) atomicMax(B.n_colors, top);
}

__host__ __device__ __forceinline__ size_t phase3_smem_bytes(int W) {
    return size_t(kChunk) * W * 4 + size_t(kChunk) * kChunkWords * 4 + kChunk * 4 + size_t(64) * W * 4 + W * 4;
}

}  // namespace grb
