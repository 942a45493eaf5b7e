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
//   * once per run, every net's marked cells and query points are written to
//     flat lists in order-position order (k_flat_*), tagged with the net's
//     position inside a chunk, so each per-chunk step below is one balanced,
//     coalesced pass over a contiguous range;
//   * cellmask holds one bit per batch ("colour") already marking each cell,
//     plane-major (colour word w of all cells contiguous);
//   * nets are processed in chunks of CH (1024, or 512 when the solver's
//     shared memory for the colour words would not fit) in order; per chunk:
//       1. raster: every mark on a query point of this chunk or (persistent
//          form) of the two chunks after it (per-cell chunk bits,
//          L2-resident, filter the rest) ORs its net's bit into the
//          chunk-local mask of the cell (five buffers by chunk index);
//       2. gather: every query point ORs, into its net's column of the chunk
//          tables, the cell's colours (forbidden batches of earlier chunks),
//          the chunk-local bits of earlier nets of the chunk (predecessors),
//          and -- in the persistent form -- the bits of the previous chunk's
//          nets and the colours of the nets two chunks back;
//       3. solve: one CTA solves first-fit inside the chunk by Jacobi
//          iteration over the predecessor DAG (converges to the unique
//          sequential solution), then applies batch capacities in order;
//       4. publish: every mark ORs its net's colour into cellmask; the
//          chunk-local mask is emptied at the chunk's query points.
//   Positions inside the batches come from a stable counting pass after the
//   run.  Plain form: one launch per step per chunk.  Persistent form: one
//   cooperative kernel in which CTA 0 solves chunk r while the other CTAs, in
//   one phase and one grid barrier, publish chunk r-1, gather chunk r+1 and
//   raster chunk r+2; the gather reads cellmask as of chunk r-2 at least (chunk
//   r-1's publish runs beside it), resolves chunk r-1's nets through that
//   chunk's local mask and its solved colours, and takes chunk r's colours
//   through the previous-chunk bits, which the solver resolves from the colours
//   it keeps in shared memory.  The solver and the other CTAs hand chunks over
//   through two monotone counters (bounded waits), so the solve never waits
//   for a publish.
#pragma once
#include "common.cuh"

namespace grb {

// Nets per chunk: CH = 512 or 1024 (== threads of the solve CTA), a template
// parameter of every per-chunk step; storage is sized for the larger.
constexpr int kChunkMax = 1024;
constexpr int kChunkMaxWords = kChunkMax / 32;

struct BatchState {
    int X, Y, n, limit, sparsity, W;   // W: colour words per cell
    const int* order;
    const int* point_off; const int* points;
    const int* hseg_off; const int* hsegs;
    const int* vseg_off; const int* vsegs;
    // Flat lists by order position (k_flat_*).
    long long* mark_off;        // [n+1]
    unsigned* mark_cell;        // cells marked by the nets (duplicates allowed)
    unsigned short* mark_jj;    // position of the marking net inside its chunk
    long long* pt_off;          // [n+1]
    unsigned* pt_cell;          // query points
    unsigned short* pt_jj;
    unsigned* cellmask;         // [W][X*Y]: word w of every cell contiguous, so the
                                // colour ORs of consecutive cells share sectors
    unsigned* localmask[5];     // [X*Y][CH/32], chunk k in buffer k % 5
    unsigned* ptchunk;          // [X*Y] bit k % 32: the cell is a query point of chunk k
    unsigned* fmask;            // [2][W][CH] forbidden colours, by chunk parity
    unsigned* pred;             // [2][CH/32][CH] predecessors inside the chunk
    unsigned* prevp;            // [2][CH/32][CH] marking nets of the previous chunk
    unsigned* fullmask;         // [W]
    int* count;                 // [32*W]
    int* n_colors;              // [1]
    int* batch_of;              // [n] colour per order position
    int* rank;                  // [n] position inside its batch
    unsigned* solved;           // [1] chunks solved (persistent form)
    int* error;
    int* error_info;
};

__device__ __forceinline__ void batch_error(const BatchState& B, int code, int info) {
    if (atomicCAS(B.error, 0, code) == 0) *B.error_info = info;
}

// Cells of the segments [s0, s1) of `segs` with step `step`, visited by the 32
// lanes of a warp: lanes fetch 32 segment endpoints per memory round trip and
// broadcast them by shuffle.  f(cell, k, cnt) gets each cell with its index
// k < cnt inside the segment; done(cnt) runs on every lane after a segment.
template <class F, class D>
__device__ __forceinline__ void warp_segment_cells(const int* segs, int s0, int s1, int step, F f, D done) {
    const int lane = threadIdx.x & 31;
    for (int base = s0; base < s1; base += 32) {
        int a = 0, b = -1;
        if (base + lane < s1) { a = segs[2 * (base + lane)]; b = segs[2 * (base + lane) + 1]; }
        const int m = min(32, s1 - base);
        for (int q = 0; q < m; ++q) {
            const int aq = __shfl_sync(0xffffffffu, a, q), bq = __shfl_sync(0xffffffffu, b, q);
            if (bq < aq) continue;
            const int cnt = (bq - aq) / step + 1;
            for (int k = lane; k < cnt; k += 32) f(aq + k * step, k, cnt);
            done(cnt);
        }
    }
}

// The (up to) four cells a query point marks: left, below, itself, right.
__device__ __forceinline__ bool point_mark(const BatchState& B, int p, int which, int* cell) {
    const int x = p / B.Y, y = p - x * B.Y;
    int cx = x, cy = y;
    if (which == 0) cx = x - 1;
    else if (which == 1) cy = y - 1;
    else if (which == 3) cx = x + 1;
    *cell = cx * B.Y + cy;
    return cx >= 0 && cx < B.X && cy >= 0;
}

// Warp per order position: number of marks and query points of its net.
__device__ __forceinline__ void flat_count(const BatchState& B, int p) {
    const int lane = threadIdx.x & 31;
    const int id = B.order[p];
    long long marks = 0;
    warp_segment_cells(B.hsegs, B.hseg_off[id], B.hseg_off[id + 1], B.sparsity * B.Y, [](int, int, int) {},
                       [&](int cnt) { marks += cnt; });
    warp_segment_cells(B.vsegs, B.vseg_off[id], B.vseg_off[id + 1], B.sparsity, [](int, int, int) {},
                       [&](int cnt) { marks += cnt; });
    const int p0 = B.point_off[id], np = B.point_off[id + 1] - p0;
    int own = 0;
    for (int k = lane; k < 4 * np; k += 32) {
        int cell;
        own += point_mark(B, B.points[p0 + k / 4], k & 3, &cell) ? 1 : 0;
    }
    for (int o = 16; o; o >>= 1) own += __shfl_xor_sync(0xffffffffu, own, o);
    if (lane == 0) {
        B.mark_off[p] = marks + own;
        B.pt_off[p] = np;
    }
}

// Warp per order position: writes its net's marks and query points at the
// (scanned) offsets.
__device__ __forceinline__ void flat_fill(const BatchState& B, int p) {
    const int lane = threadIdx.x & 31;
    const int id = B.order[p];
    // Position inside a chunk of kChunkMax; reduced mod CH where read.
    const unsigned short jj = static_cast<unsigned short>(p % kChunkMax);
    long long o = B.mark_off[p];
    auto put = [&](int cell, int k, int) {
        B.mark_cell[o + k] = static_cast<unsigned>(cell);
        B.mark_jj[o + k] = jj;
    };
    auto advance = [&](int cnt) { o += cnt; };
    warp_segment_cells(B.hsegs, B.hseg_off[id], B.hseg_off[id + 1], B.sparsity * B.Y, put, advance);
    warp_segment_cells(B.vsegs, B.vseg_off[id], B.vseg_off[id + 1], B.sparsity, put, advance);
    const int p0 = B.point_off[id], np = B.point_off[id + 1] - p0;
    for (int base = 0; base < 4 * np; base += 32) {
        const int k = base + lane;
        int cell = 0;
        const bool ok = k < 4 * np && point_mark(B, B.points[p0 + k / 4], k & 3, &cell);
        const unsigned ball = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const long long at = o + __popc(ball & ((1u << lane) - 1u));
            B.mark_cell[at] = static_cast<unsigned>(cell);
            B.mark_jj[at] = jj;
        }
        o += __popc(ball);
    }
    const long long q = B.pt_off[p];
    for (int k = lane; k < np; k += 32) {
        B.pt_cell[q + k] = static_cast<unsigned>(B.points[p0 + k]);
        B.pt_jj[q + k] = jj;
    }
}

constexpr int kLocalMasks = 5;
__device__ __forceinline__ unsigned* chunk_mask(const BatchState& B, int chunk) { return B.localmask[chunk % kLocalMasks]; }

// Query-point bits of the chunk at s: bit (chunk % 32) of every query point
// cell of the chunk is set (set) or cleared.
template <int CH>
__device__ __forceinline__ void batch_point_bits(const BatchState& B, int s, bool set, long long t, long long nt) {
    const int m = min(CH, B.n - s);
    const unsigned bit = 1u << ((s / CH) & 31);
    const long long a = B.pt_off[s], b = B.pt_off[s + m];
    for (long long k = a + t; k < b; k += nt) {
        unsigned* w = B.ptchunk + __ldg(B.pt_cell + k);
        if (set) red_or(w, bit);
        else asm volatile("red.relaxed.gpu.global.and.b32 [%0], %1;" ::"l"(w), "r"(~bit) : "memory");
    }
}

// Step 1: the chunk at order position s rasters its marks.  Only a cell that
// is a query point of this chunk or of the `ahead` chunks after it is ever
// read back, so the raster keeps the marks whose cell has one of those
// query-point bits; the bits live in a 4-byte-per-cell array that stays in L2,
// the chunk-local masks do not.  Threads t of nt.
template <int CH>
__device__ __forceinline__ void batch_raster(const BatchState& B, int s, int ahead, long long t, long long nt) {
    const int m = min(CH, B.n - s), chunk = s / CH;
    unsigned want = 0u;
    for (int a = 0; a <= ahead; ++a) want |= 1u << ((chunk + a) & 31);
    unsigned* lm = chunk_mask(B, chunk);
    const long long a = B.mark_off[s], b = B.mark_off[s + m];
    // Four marks per thread and pass, every load of a pass issued first.
    for (long long k0 = a + t; k0 < b; k0 += 4 * nt) {
        unsigned q[4], bits[4];
        int jj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long k = k0 + u * nt;
            q[u] = k < b ? __ldg(B.mark_cell + k) : 0u;
            jj[u] = k < b ? (__ldg(B.mark_jj + k) & (CH - 1)) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) bits[u] = jj[u] >= 0 ? __ldcg(B.ptchunk + q[u]) : 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (bits[u] & want) red_or(lm + size_t(q[u]) * (CH / 32) + (jj[u] >> 5), 1u << (jj[u] & 31));
    }
}

// The chunk-local mask of the chunk at s is nonzero only at query points of
// this chunk and the `ahead` chunks after it: zero the whole record of each of
// those cells.
template <int CH>
__device__ __forceinline__ void batch_clear(const BatchState& B, int s, int ahead, long long t, long long nt) {
    unsigned* lm = chunk_mask(B, s / CH);
    const long long a = B.pt_off[s];
    const long long b = B.pt_off[min(s + (ahead + 1) * CH, B.n)];
    constexpr int kParts = (CH / 32) / 4;  // 16-byte groups of a record
    const long long items = (b - a) * kParts;
    for (long long k = t; k < items; k += nt) {
        const long long pi = a + k / kParts;
        const int part = int(k % kParts);
        uint4* rec = reinterpret_cast<uint4*>(lm + size_t(__ldg(B.pt_cell + pi)) * (CH / 32));
        rec[part] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Step 2: per query point, OR into the net's columns the cell's colours, the
// earlier nets' bits of this chunk and, with lookback >= 1, the bits of the
// previous chunk's nets (resolved by the solver, which knows their colours);
// with lookback 2 also the colours of the nets two chunks back that mark the
// cell (that chunk is solved, its colours published or being published).
// Each item is a 16-byte group of one record (W and (CH / 32) are
// multiples of 4).
template <int CH>
__device__ __forceinline__ void batch_gather(const BatchState& B, int s, int lookback, long long t, long long nt) {
    const int chunk = s / CH, m = min(CH, B.n - s), W = B.W;
    const unsigned* lm = chunk_mask(B, chunk);
    const unsigned* lp = lookback >= 1 ? chunk_mask(B, chunk - 1) : nullptr;
    const unsigned* lp2 = lookback >= 2 ? chunk_mask(B, chunk - 2) : nullptr;
    unsigned* F = B.fmask + size_t(chunk & 1) * W * CH;
    unsigned* P = B.pred + size_t(chunk & 1) * (CH / 32) * CH;
    unsigned* Q = B.prevp + size_t(chunk & 1) * (CH / 32) * CH;
    const int gw = W / 4, gl = (CH / 32) / 4;
    const int per = gw + gl * (1 + lookback);
    const long long a = B.pt_off[s], b = B.pt_off[s + m];
    const long long items = (b - a) * per;
    for (long long k = t; k < items; k += nt) {
        const long long pi = k / per;
        const int g = int(k - pi * per);
        const unsigned q = __ldg(B.pt_cell + a + pi);
        const int jj = __ldg(B.pt_jj + a + pi) & (CH - 1);
        uint4 v;
        unsigned* dst;
        int w0;
        if (g < gw) {
            w0 = 4 * g;
            const size_t XY = size_t(B.X) * B.Y;
            v.x = __ldcg(B.cellmask + (4 * g) * XY + q);
            v.y = __ldcg(B.cellmask + (4 * g + 1) * XY + q);
            v.z = __ldcg(B.cellmask + (4 * g + 2) * XY + q);
            v.w = __ldcg(B.cellmask + (4 * g + 3) * XY + q);
            dst = F;
        } else if (g < gw + gl) {
            w0 = 4 * (g - gw);
            if (w0 > (jj >> 5)) continue;
            v = __ldcg(reinterpret_cast<const uint4*>(lm + size_t(q) * (CH / 32)) + (g - gw));
            const unsigned own = (1u << (jj & 31)) - 1u;  // earlier nets of the own word
            const int ow = (jj >> 5) - w0;
            if (ow == 0) { v.x &= own; v.y = v.z = v.w = 0u; }
            else if (ow == 1) { v.y &= own; v.z = v.w = 0u; }
            else if (ow == 2) { v.z &= own; v.w = 0u; }
            else if (ow == 3) v.w &= own;
            dst = P;
        } else if (g < gw + 2 * gl) {
            w0 = 4 * (g - gw - gl);
            v = __ldcg(reinterpret_cast<const uint4*>(lp + size_t(q) * (CH / 32)) + (g - gw - gl));
            dst = Q;
        } else {
            w0 = 4 * (g - gw - 2 * gl);
            v = __ldcg(reinterpret_cast<const uint4*>(lp2 + size_t(q) * (CH / 32)) + (g - gw - 2 * gl));
            const unsigned vw[4] = {v.x, v.y, v.z, v.w};
            const int* col2 = B.batch_of + size_t(chunk - 2) * CH;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                for (unsigned bits = vw[u]; bits; bits &= bits - 1) {
                    const int c = __ldcg(col2 + (w0 + u) * 32 + __ffs(bits) - 1);
                    red_or(F + size_t(c >> 5) * CH + jj, 1u << (c & 31));
                }
            continue;
        }
        if (v.x) red_or(dst + size_t(w0) * CH + jj, v.x);
        if (v.y) red_or(dst + size_t(w0 + 1) * CH + jj, v.y);
        if (v.z) red_or(dst + size_t(w0 + 2) * CH + jj, v.z);
        if (v.w) red_or(dst + size_t(w0 + 3) * CH + jj, v.w);
    }
}

// Step 4: the chunk at s publishes its colours.
template <int CH>
__device__ __forceinline__ void batch_publish(const BatchState& B, int s, long long t, long long nt) {
    const int m = min(CH, B.n - s);
    const long long a = B.mark_off[s], b = B.mark_off[s + m];
    for (long long k = a + t; k < b; k += nt) {
        const unsigned q = __ldg(B.mark_cell + k);
        const int jj = __ldg(B.mark_jj + k) & (CH - 1);
        const int c = __ldcg(B.batch_of + s + jj);
        red_or(B.cellmask + size_t(c >> 5) * B.X * B.Y + q, 1u << (c & 31));
    }
}

// Shared memory of the solving CTA (kept across chunks in the persistent form).
struct SolveSmem {
    unsigned* U;     // [W][CH] colours a net may not take (published, full, previous chunk)
    unsigned* P;     // [(CH / 32)][CH] predecessor bits
    int* col;        // [CH] colour of each net of the chunk
    int* colp;       // [CH] colours of the previous chunk
    int* cnt;        // [32W] nets per colour so far
    int* wh;         // [CH/32][32W] per-warp colour counts (zero between uses), or
                     // for W > kWarpCountWords a [32W] running count
    bool per_warp;   // wh holds per-warp counts
    unsigned* full;  // [W] colours whose batch is full
};

// Up to this many colour words the ranks use per-warp colour counts (three
// barriers); beyond it, warps add their counts in turn (one barrier per warp).
constexpr int kWarpCountWords = 32;

// Shared memory a solving CTA may use (the per-warp colour counts are dropped
// for the running count when they do not fit).
constexpr size_t kSolveSmemLimit = 220 * 1024;
template <int CH>
__host__ __device__ __forceinline__ size_t solve_smem_base(int W) {
    const size_t C = 32 * size_t(W);
    return size_t(CH) * W * 4 + size_t(CH) * (CH / 32) * 4 + 2 * size_t(CH) * 4 + C * 4 + size_t(W) * 4;
}
template <int CH>
__host__ __device__ __forceinline__ bool solve_per_warp(int W) {
    return W <= kWarpCountWords && solve_smem_base<CH>(W) + (CH / 32) * 32 * size_t(W) * 4 <= kSolveSmemLimit;
}
template <int CH>
__host__ __device__ __forceinline__ size_t solve_smem_bytes(int W) {
    const size_t C = 32 * size_t(W);
    const size_t wh = solve_per_warp<CH>(W) ? (CH / 32) * C : C;
    return size_t(CH) * W * 4 + size_t(CH) * (CH / 32) * 4 + 2 * size_t(CH) * 4 + C * 4 + wh * 4 +
           size_t(W) * 4;
}

template <int CH>
__device__ __forceinline__ SolveSmem solve_smem(unsigned* base, int W) {
    const int C = 32 * W;
    SolveSmem S;
    S.U = base;
    S.P = S.U + size_t(CH) * W;
    S.col = reinterpret_cast<int*>(S.P + size_t(CH) * (CH / 32));
    S.colp = S.col + CH;
    S.cnt = S.colp + CH;
    S.wh = S.cnt + C;
    S.per_warp = solve_per_warp<CH>(W);
    S.full = reinterpret_cast<unsigned*>(S.wh + (S.per_warp ? (CH / 32) * C : C));
    return S;
}

// The smallest colour c >= c0 net `tid` may take: not in U, not held by a
// predecessor (pmask: which predecessor words are nonzero).  C if none.
// Word by word from c0's: the word's forbidden bits are U's plus the colours
// of the predecessors that fall in it (one pass over the predecessors per
// word, whatever the number of colours the net has to skip).
template <int CH>
__device__ __forceinline__ int first_fit(const SolveSmem& S, int tid, int W, unsigned pmask, int c0) {
    for (int w = c0 >> 5; w < W; ++w) {
        unsigned used = S.U[w * CH + tid];
        if (w == (c0 >> 5)) used |= (1u << (c0 & 31)) - 1u;
        if (used == 0xffffffffu) continue;
        for (unsigned pm = pmask; pm; pm &= pm - 1) {
            const int pw = __ffs(pm) - 1;
            unsigned bits = S.P[pw * CH + tid];
            while (bits) {
                const int ci = S.col[pw * 32 + __ffs(bits) - 1];
                bits &= bits - 1;
                if ((ci >> 5) == w) used |= 1u << (ci & 31);  // ci = -1 (not yet coloured) is in no word
            }
        }
        if (used != 0xffffffffu) return w * 32 + __ffs(~used) - 1;
    }
    return 32 * W;
}

// The solve runs on threads 0..CH-1 of its CTA and synchronises them
// with named barrier 1 (the CTA may hold more threads, which do not take part).
template <int CH>
__device__ __forceinline__ void solve_sync() { asm volatile("bar.sync 1, %0;" ::"n"(CH) : "memory"); }
template <int CH>
__device__ __forceinline__ bool solve_sync_or(bool v) {
    int r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.s32 p, %1, 0;\n bar.red.or.pred q, 1, %2, p;\n selp.s32 %0, 1, 0, q;\n}"
        : "=r"(r) : "r"(int(v)), "n"(CH) : "memory");
    return r != 0;
}

// Step 3 (threads 0..CH-1 of a CTA): first-fit of the chunk at order
// position s.  S.cnt and S.full hold the state of the chunks before it;
// with `lookback`, S.colp holds the previous chunk's colours.  The chunk's
// tables are read once and cleared for reuse by chunk s + 2 * CH.
// Returns false on colour overflow (kELimit recorded).
template <int CH>
__device__ __forceinline__ bool batch_solve(const BatchState& B, int s, bool lookback, const SolveSmem& S) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int chunk = s / CH, m = min(CH, B.n - s);
    const int W = B.W, C = 32 * W;
    unsigned* Fg = B.fmask + size_t(chunk & 1) * W * CH;
    unsigned* Pg = B.pred + size_t(chunk & 1) * (CH / 32) * CH;
    unsigned* Qg = B.prevp + size_t(chunk & 1) * (CH / 32) * CH;
    __shared__ int first_bad, overflow;
    if (tid == 0) overflow = 0;
    unsigned pmask = 0;
    int c0 = 0;  // first colour not in U
    if (tid < m) {
        // Every load of a group is issued before its stores, so the round
        // trips overlap (the tables were just written by other SMs).
        for (int w0 = 0; w0 < W; w0 += 8) {
            unsigned v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = w0 + k < W ? __ldcg(Fg + size_t(w0 + k) * CH + tid) : 0u;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (w0 + k >= W) break;
                if (v[k]) Fg[size_t(w0 + k) * CH + tid] = 0u;
                S.U[(w0 + k) * CH + tid] = v[k] | S.full[w0 + k];
            }
        }
        {
            unsigned v[(CH / 32)];
#pragma unroll
            for (int w = 0; w < (CH / 32); ++w) v[w] = w <= (tid >> 5) ? __ldcg(Pg + w * CH + tid) : 0u;
#pragma unroll
            for (int w = 0; w < (CH / 32); ++w) {
                S.P[w * CH + tid] = v[w];
                if (v[w]) { Pg[w * CH + tid] = 0u; pmask |= 1u << w; }
            }
        }
        if (lookback) {
            unsigned v[(CH / 32)];
#pragma unroll
            for (int w = 0; w < (CH / 32); ++w) v[w] = __ldcg(Qg + w * CH + tid);
#pragma unroll
            for (int w = 0; w < (CH / 32); ++w) {
                unsigned bits = v[w];
                if (bits) Qg[w * CH + tid] = 0u;
                while (bits) {
                    const int c = S.colp[w * 32 + __ffs(bits) - 1];
                    bits &= bits - 1;
                    S.U[(c >> 5) * CH + tid] |= 1u << (c & 31);
                }
            }
        }
        c0 = first_fit<CH>(S, tid, W, 0u, 0);
    }
    S.col[tid] = -1;
    solve_sync<CH>();
    int fixed = 0;  // nets below `fixed` are final
    int rank = 0;
    bool counted = false;  // this chunk's nets are in S.cnt already
    __shared__ int tight;
    while (true) {
        // Jacobi sweeps until the colouring is a fixed point.
        while (true) {
            int mine = tid < m ? S.col[tid] : -1;
            if (tid < m && tid >= fixed) {
                mine = first_fit<CH>(S, tid, W, pmask, c0);
                if (mine >= C) { overflow = 1; mine = C - 1; }
            }
            solve_sync<CH>();
            const bool changed = tid < m && S.col[tid] != mine;
            if (tid < m) S.col[tid] = mine;
            if (!solve_sync_or<CH>(changed)) break;
        }
        if (overflow) break;
        // Position of every net inside its batch, in chunk order: colour
        // counts of the earlier warps plus the rank inside the own warp.
        if (tid == 0) first_bad = m;
        const int c = tid < m ? S.col[tid] : -1 - lane;  // distinct dummies for idle lanes
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const bool leader = tid < m && lane == __ffs(peers) - 1;
        const int within = __popc(peers & ((1u << lane) - 1u));
        if (S.per_warp) {
            if (leader) S.wh[warp * C + c] = __popc(peers);
            solve_sync<CH>();
            if (tid < m) {
                int r = S.cnt[c] + within;
                for (int w = 0; w < warp; ++w) r += S.wh[w * C + c];
                rank = r;
                if (r >= B.limit) atomicMin(&first_bad, tid);
            }
            solve_sync<CH>();
            if (leader) S.wh[warp * C + c] = 0;
        } else {
            // Per-colour totals first: while no batch reaches the limit, no
            // position inside a batch is needed here (the rank pass after the
            // run assigns them); else warps add their counts in turn.
            if (tid == 0) tight = 0;
            solve_sync<CH>();
            if (leader && atomicAdd(S.cnt + c, __popc(peers)) + __popc(peers) > B.limit) tight = 1;
            solve_sync<CH>();
            if (!tight) {
                counted = true;
            } else {
                if (leader) atomicSub(S.cnt + c, __popc(peers));
                solve_sync<CH>();
                for (int k = tid; k < C; k += CH) S.wh[k] = S.cnt[k];
                solve_sync<CH>();
                for (int w = 0; w < (m + 31) / 32; ++w) {
                    if (warp == w && tid < m) {
                        rank = S.wh[c] + within;
                        if (leader) S.wh[c] += __popc(peers);
                        if (rank >= B.limit) atomicMin(&first_bad, tid);
                    }
                    solve_sync<CH>();
                }
            }
        }
        const int bad = first_bad;
        if (bad >= m) {
            if (leader && !counted) atomicAdd(S.cnt + c, __popc(peers));
            break;
        }
        // Net `bad` finds its colour full; so does every later net.
        const int fc = S.col[bad];
        if (tid == 0) S.full[fc >> 5] |= 1u << (fc & 31);
        if (tid >= bad && tid < m) {
            S.U[(fc >> 5) * CH + tid] |= 1u << (fc & 31);
            c0 = first_fit<CH>(S, tid, W, 0u, c0);
        }
        fixed = bad;
        solve_sync<CH>();
    }
    if (overflow) {
        if (tid == 0) batch_error(B, kELimit, s);
        return false;
    }
    int top = 0;
    if (tid < m) {
        const int c = S.col[tid];
        B.batch_of[s + tid] = c;
        S.colp[tid] = c;
        top = c + 1;
    }
    for (int o = 16; o; o >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
    if (lane == 0 && top) atomicMax(B.n_colors, top);
    solve_sync<CH>();
    return true;
}

}  // namespace grb
