// zshape.cuh -- Z-shape stage: two-bend candidates on projection planes,
// layer-range DP per tree node and traceback; bounding-box batch refinement.
//
// Semantics of the reference's Z-shape pipeline (zshape.cuh:5-404,
// zshape_topology.hpp:7-57 and 249-290).  All costs are int32: a wire costs
// |presum[a] - presum[b]| clamped to 5e8, a via clamp(vcost, 1, 1e6), with 1e9
// as infinity; sums wrap as 32-bit integers exactly as the device code does.
// Planes of LAYER = L+1 layers of N x N (N = max(X, Y)) hold, per 2-D position
// and layer: map 0 = node DP, 1..3 = best arrival of child slot j, 4 = the
// current edge's candidate rows and columns, 5 = chosen layer per node; prev
// 0..5 the matching back-pointers, prev 11..13 the turn cells of slot j.
// A position on GGR layer i sits at i*N*N + (x*N + y) when ((i & 1) ^ D) is 1,
// at i*N*N + (y*N + x) otherwise, D = DIR ^ 1; GGR layer i is routing layer
// i-1 (layer 0 carries no wires and costs an infinite via).
//
// B200 form: one CTA per net (the reference uses one warp); a bounding-box
// batch holds at most 250 nets, so a whole CTA per net keeps the GPU busy and
// splits a long edge's row/column relaxations and via sweeps over all its
// threads.  The nets of a batch have disjoint bounding boxes, so their plane
// cells never overlap.  Warp 0 runs the node DP (one lane per lower layer,
// then one per layer); thread 0 runs the traceback in the reference's order
// and converts each segment straight into route words (convert_routes).
#pragma once
#include "commit.cuh"
#include "common.cuh"

namespace grb {

constexpr int kZInf = 1000000000;  // zshape.cuh:6

struct ZTrees {
    const int* node_off;  // [n+1] by net id
    const int* pos;       // per node: x*N + y
    const int* pin;       // per node: pin layer + 1, -1 for Steiner points
    const int* child;     // [3 per node] net-local preorder index, -1 = none
    int* map;             // 6 planes
    int* prev;            // 16 planes
    int N, LAYER, D;
    long long NN, LNN;
};

__device__ __forceinline__ int zadd(int a, int b) {
    return static_cast<int>(static_cast<unsigned>(a) + static_cast<unsigned>(b));
}
__device__ __forceinline__ int zidx(const ZTrees& Z, int i, int x, int y) {
    return static_cast<int>(i * Z.NN + (((i & 1) ^ Z.D) ? x * Z.N + y : y * Z.N + x));
}
// ViaCosts (zshape.cuh:20-31) and boundedWireCost over WireCosts
// (zshape.cuh:8-19, 32-35) for plane layer i (1..L, routing layer i-1) at grid
// positions.  The reference decodes (layer, x, y) from a plane index; the
// loops here know the positions and read the same cells directly.
__device__ __forceinline__ int zvia_at(const Tables& T, int i, int x, int y) {
    return static_cast<int>(fminf(fmaxf(T.vcost[cell_index(T, i - 1, x, y)], 1.f), 1.e6f));
}
__device__ __forceinline__ int zwire_at(const Tables& T, int i, int x0, int y0, int x1, int y1) {
    return static_cast<int>(fmin(fabs(T.presum[cell_index(T, i - 1, x0, y0)] - T.presum[cell_index(T, i - 1, x1, y1)]),
                                 static_cast<double>(kZInf / 2)));
}

// viaSweep (zshape.cuh:42-61) on plane 4 at 2-D position (x, y): up, then
// down.  The position's layer column is loaded into registers first, so the
// two dependent chains run without a memory round trip per layer.
__device__ __noinline__ void zvia_sweep(const Tables& T, const ZTrees& Z, int x, int y) {
    constexpr int K = kMaxLayers + 1;
    int* m = Z.map + 4 * Z.LNN;
    int* p = Z.prev + 4 * Z.LNN;
    int* p5 = Z.prev + 5 * Z.LNN;
    int mv[K], pv[K], vc[K], q[K];  // q: layer of the cell the value came from
#pragma unroll
    for (int i = 1; i < K; ++i) {
        if (i < Z.LAYER) {
            const int c = zidx(Z, i, x, y);
            mv[i] = m[c];
            pv[i] = p[c];
            vc[i] = zvia_at(T, i, x, y);
            q[i] = i;
        }
    }
#pragma unroll
    for (int i = 2; i < K; ++i) {
        if (i < Z.LAYER) {
            const int v = zadd(mv[i - 1], vc[i - 1]);
            if (mv[i] > v) { mv[i] = v; pv[i] = pv[i - 1]; q[i] = i - 1; }
        }
    }
#pragma unroll
    for (int i = K - 2; i >= 1; --i) {
        if (i <= Z.LAYER - 2) {
            const int v = zadd(mv[i + 1], vc[i]);
            if (mv[i] > v) { mv[i] = v; pv[i] = pv[i + 1]; q[i] = i + 1; }
        }
    }
#pragma unroll
    for (int i = 1; i < K; ++i) {
        if (i < Z.LAYER) {
            const int c = zidx(Z, i, x, y);
            m[c] = mv[i];
            p[c] = pv[i];
            p5[c] = zidx(Z, q[i], x, y);
        }
    }
}

// The (layer, position) items of an edge phase over plane layers 1..LAYER-1:
// the layers along y ((i & 1) ^ D) come first, `ey` positions each, then the
// others, `ex` positions each.  Flattening the layers into one index space
// gives a layer's items to different threads: the reference's loop over the
// layers (one dependent load chain per layer and thread) becomes a single pass.
struct ZItems {
    int ey, ex, ny, nx, iy, ix;  // extents, layer counts, first layer of each kind
    __device__ int count() const { return ny * ey + nx * ex; }
};
__device__ __forceinline__ ZItems zitems(const ZTrees& Z, int ey, int ex) {
    ZItems I;
    I.ey = ey; I.ex = ex;
    I.iy = 1 + Z.D;
    I.ix = 2 - Z.D;
    I.ny = I.iy <= Z.LAYER - 1 ? (Z.LAYER - 1 - I.iy) / 2 + 1 : 0;
    I.nx = I.ix <= Z.LAYER - 1 ? (Z.LAYER - 1 - I.ix) / 2 + 1 : 0;
    return I;
}
// Item k -> plane layer i, offset o along its box side, along-y flag.
__device__ __forceinline__ void zitem(const ZItems& I, int k, int& i, int& o, bool& ay) {
    const int ky = I.ny * I.ey;
    ay = k < ky;
    if (ay) { i = I.iy + 2 * (k / I.ey); o = k % I.ey; }
    else { k -= ky; i = I.ix + 2 * (k / I.ex); o = k % I.ex; }
}
// Items a thread takes per pass, their loads issued together: 1 measured
// fastest (1,387 ms for the persistent stage at the 900K-net design against
// 1,421 with 2 and 1,502 with 4, which spill in the persistent kernel).
constexpr int kZUnroll = 1;

// Child slot j (1..3) of node (tox, toy): fill plane j at the node from the
// child at (fromx, fromy) (zshape.cuh:87-237).
__device__ __forceinline__ void zedge(const Tables& T, const ZTrees& Z, int j, int fromx, int fromy, int tox, int toy,
                                      int lane, int nth) {
    const int LAYER = Z.LAYER, D = Z.D;
    const long long NN = Z.NN;
    int* map0 = Z.map;
    int* m4 = Z.map + 4 * Z.LNN;
    int* p4 = Z.prev + 4 * Z.LNN;
    int* p5 = Z.prev + 5 * Z.LNN;
    int* mj = Z.map + j * Z.LNN;
    int* pj = Z.prev + j * Z.LNN;
    int* p2j = Z.prev + (10 + j) * Z.LNN;
    const int minx = min(fromx, tox), maxx = max(fromx, tox), miny = min(fromy, toy), maxy = max(fromy, toy);
    if (fromx != tox && fromy != toy) {
        // Clear the candidate rows and columns of the edge's box.
        for (int a = minx + lane; a <= maxx; a += nth)
            for (int i = 1; i < LAYER; ++i) {
                if ((i & 1) ^ D) { m4[i * NN + a * Z.N + toy] = kZInf; m4[i * NN + a * Z.N + fromy] = kZInf; }
                else { m4[i * NN + toy * Z.N + a] = kZInf; m4[i * NN + fromy * Z.N + a] = kZInf; }
            }
        for (int b = miny + lane; b <= maxy; b += nth)
            for (int i = 1; i < LAYER; ++i) {
                if ((i & 1) ^ D) { m4[i * NN + tox * Z.N + b] = kZInf; m4[i * NN + fromx * Z.N + b] = kZInf; }
                else { m4[i * NN + b * Z.N + tox] = kZInf; m4[i * NN + b * Z.N + fromx] = kZInf; }
            }
        __syncthreads();
        // Straight runs out of the child along each layer's direction.
        {
            const ZItems I = zitems(Z, maxy - miny + 1, maxx - minx + 1);
            const int items = I.count();
            for (int k0 = lane; k0 < items; k0 += kZUnroll * nth) {
                int cur[kZUnroll], last[kZUnroll], base[kZUnroll], w[kZUnroll];
                bool ok[kZUnroll];
#pragma unroll
                for (int u = 0; u < kZUnroll; ++u) {
                    const int k = k0 + u * nth;
                    ok[u] = false;
                    if (k >= items) continue;
                    int i, o;
                    bool ay;
                    zitem(I, k, i, o, ay);
                    const int b = (ay ? miny : minx) + o;
                    if (b == (ay ? fromy : fromx)) continue;
                    ok[u] = true;
                    if (ay) {
                        last[u] = static_cast<int>(i * NN + fromx * Z.N + fromy);
                        cur[u] = static_cast<int>(i * NN + fromx * Z.N + b);
                        w[u] = zwire_at(T, i, fromx, fromy, fromx, b);
                    } else {
                        last[u] = static_cast<int>(i * NN + fromy * Z.N + fromx);
                        cur[u] = static_cast<int>(i * NN + fromy * Z.N + b);
                        w[u] = zwire_at(T, i, fromx, fromy, b, fromy);
                    }
                    base[u] = map0[last[u]];
                }
#pragma unroll
                for (int u = 0; u < kZUnroll; ++u)
                    if (ok[u]) { m4[cur[u]] = zadd(base[u], w[u]); p4[cur[u]] = last[u]; }
            }
        }
        __syncthreads();
        // Layer changes on the child's column and row (distinct positions).
        {
            const int ncol = maxy - miny + 1;
            for (int k = lane; k < ncol + (maxx - minx + 1); k += nth) {
                if (k < ncol) { const int b = miny + k; if (b != fromy) zvia_sweep(T, Z, fromx, b); }
                else { const int b = minx + (k - ncol); if (b != fromx) zvia_sweep(T, Z, b, fromy); }
            }
        }
        __syncthreads();
        // Cross the box to the node's row / column (layers along y cross at
        // every column of the box, the others at every row).
        {
            const ZItems I = zitems(Z, maxx - minx + 1, maxy - miny + 1);
            const int items = I.count();
            for (int k0 = lane; k0 < items; k0 += kZUnroll * nth) {
                int cur[kZUnroll], last[kZUnroll], v[kZUnroll], mc[kZUnroll], pl[kZUnroll];
                bool ok[kZUnroll];
#pragma unroll
                for (int u = 0; u < kZUnroll; ++u) {
                    const int k = k0 + u * nth;
                    ok[u] = k < items;
                    if (!ok[u]) continue;
                    int i, o;
                    bool ay;
                    zitem(I, k, i, o, ay);
                    int w;
                    if (ay) {
                        const int b = minx + o;
                        last[u] = static_cast<int>(i * NN + b * Z.N + fromy);
                        cur[u] = static_cast<int>(i * NN + b * Z.N + toy);
                        w = zwire_at(T, i, b, fromy, b, toy);
                    } else {
                        const int b = miny + o;
                        last[u] = static_cast<int>(i * NN + b * Z.N + fromx);
                        cur[u] = static_cast<int>(i * NN + b * Z.N + tox);
                        w = zwire_at(T, i, fromx, b, tox, b);
                    }
                    v[u] = zadd(m4[last[u]], w);
                    mc[u] = m4[cur[u]];
                    pl[u] = p4[last[u]];
                }
#pragma unroll
                for (int u = 0; u < kZUnroll; ++u)
                    if (ok[u] && v[u] < mc[u]) { m4[cur[u]] = v[u]; p4[cur[u]] = pl[u]; }
            }
        }
        __syncthreads();
        {
            const int ncol = maxy - miny + 1;
            for (int k = lane; k < ncol + (maxx - minx + 1); k += nth) {
                if (k < ncol) { const int b = miny + k; if (b != toy) zvia_sweep(T, Z, tox, b); }
                else { const int b = minx + (k - ncol); if (b != tox) zvia_sweep(T, Z, b, toy); }
            }
        }
        __syncthreads();
        // Last run into the node: per layer, the first minimum over the
        // positions of the node's row/column (the reference scans them in
        // order keeping strict improvements), as the (value, position) minimum.
        // A warp per layer (lanes over the positions, several loads in
        // flight per lane); its result goes to shared memory, and after one
        // barrier thread i applies layer i's.
        __shared__ int red_v[kMaxLayers + 1], red_b[kMaxLayers + 1];
        {
            const int warp = lane >> 5, wl = lane & 31, nw = (nth + 31) / 32;
            for (int i = 1 + warp; i < LAYER; i += nw) {
                const bool ay = ((i & 1) ^ D) != 0;
                const int lo = ay ? miny : minx, hi = ay ? maxy : maxx, skip = ay ? toy : tox;
                int bv = 0, bb = -1;
                for (int b0 = lo + wl; b0 <= hi; b0 += kZUnroll * 32) {
                    int v[kZUnroll];
                    bool ok[kZUnroll];
#pragma unroll
                    for (int u = 0; u < kZUnroll; ++u) {
                        const int b = b0 + u * 32;
                        ok[u] = b <= hi && b != skip;
                        if (!ok[u]) continue;
                        const int last = static_cast<int>(ay ? i * NN + tox * Z.N + b : i * NN + toy * Z.N + b);
                        v[u] = zadd(m4[last], ay ? zwire_at(T, i, tox, b, tox, toy) : zwire_at(T, i, b, toy, tox, toy));
                    }
#pragma unroll
                    for (int u = 0; u < kZUnroll; ++u)
                        if (ok[u] && (bb < 0 || v[u] < bv)) { bv = v[u]; bb = b0 + u * 32; }
                }
                for (int o = 16; o; o >>= 1) {
                    const int ov = __shfl_down_sync(0xffffffffu, bv, o), ob = __shfl_down_sync(0xffffffffu, bb, o);
                    if (ob >= 0 && (bb < 0 || ov < bv || (ov == bv && ob < bb))) { bv = ov; bb = ob; }
                }
                if (wl == 0) { red_v[i] = bv; red_b[i] = bb; }
            }
        }
        __syncthreads();
        if (lane >= 1 && lane < LAYER) {
            const int i = lane;
            const bool ay = ((i & 1) ^ D) != 0;
            const int cur = static_cast<int>(ay ? i * NN + tox * Z.N + toy : i * NN + toy * Z.N + tox);
            const int bv = red_v[i], bb = red_b[i];
            if (bb >= 0 && bv < mj[cur]) {
                const int last = static_cast<int>(ay ? i * NN + tox * Z.N + bb : i * NN + toy * Z.N + bb);
                mj[cur] = bv; pj[cur] = p4[last]; p2j[cur] = p5[last];
            }
        }
    } else if (fromx == tox) {
        for (int i = 1 + lane; i < LAYER; i += nth) {
            if ((i & 1) ^ D) {
                const int last = static_cast<int>(i * NN + fromx * Z.N + fromy), cur = static_cast<int>(i * NN + tox * Z.N + toy);
                const int v = zadd(map0[last], zwire_at(T, i, fromx, fromy, tox, toy));
                if (mj[cur] > v) { mj[cur] = v; pj[cur] = last; }
            } else {
                mj[i * NN + toy * Z.N + tox] = kZInf;
            }
        }
    } else {  // fromy == toy
        for (int i = 1 + lane; i < LAYER; i += nth) {
            if ((!(i & 1)) ^ D) {
                const int last = static_cast<int>(i * NN + fromy * Z.N + fromx), cur = static_cast<int>(i * NN + toy * Z.N + tox);
                const int v = zadd(map0[last], zwire_at(T, i, fromx, fromy, tox, toy));
                if (mj[cur] > v) { mj[cur] = v; pj[cur] = last; }
            } else {
                mj[i * NN + tox * Z.N + toy] = kZInf;
            }
        }
    }
    __syncthreads();
}

// Layer-range DP of one node (zshape.cuh:241-267) with the warp: lane
// `lower` walks its uppers (the
// child and via values of every layer come by shuffle) and writes each
// range's value and code to shared memory `cand` (2 * LAYER * LAYER ints);
// then lane i takes, over the allowed ranges containing layer i in the
// sequential (lower, upper) order, the first strict minimum -- exactly the
// value and code the sequential loop leaves at layer i.
__device__ __forceinline__ void znode_dp_warp(const Tables& T, const ZTrees& Z, int tox, int toy, int pin,
                                              const int* ch, int lane, int* cand) {
    const int LAYER = Z.LAYER;
    const int idx_l = lane < LAYER ? zidx(Z, lane, tox, toy) : 0;
    int pv[3];
    for (int j = 0; j < 3; ++j) pv[j] = (lane < LAYER && ch[j] != -1) ? Z.map[(j + 1) * Z.LNN + idx_l] : 0;
    const int vc = lane < LAYER ? (lane >= 1 ? zvia_at(T, lane, tox, toy) : kZInf) : 0;
    const int lower = lane;
    int viaSum = 0, minCost = kZInf, bestpos[3] = {0, 0, 0};
    int costs[3] = {ch[0] == -1 ? 0 : kZInf, ch[1] == -1 ? 0 : kZInf, ch[2] == -1 ? 0 : kZInf};
    for (int upper = 0; upper < LAYER; ++upper) {
        int v[3];
        for (int j = 0; j < 3; ++j) v[j] = __shfl_sync(0xffffffffu, pv[j], upper);
        const int vu = __shfl_sync(0xffffffffu, vc, upper);
        if (lower >= LAYER || upper < lower) continue;
        for (int j = 0; j < 3; ++j)
            if (ch[j] != -1 && v[j] < costs[j]) { costs[j] = v[j]; bestpos[j] = upper; }
        if (1LL * costs[0] + costs[1] + costs[2] < minCost) minCost = costs[0] + costs[1] + costs[2];
        const bool allowed = pin == -1 || (lower <= pin && pin <= upper);
        cand[lower * LAYER + upper] = zadd(minCost, viaSum);
        cand[LAYER * LAYER + lower * LAYER + upper] =
            allowed ? (((lower * LAYER + upper) * LAYER + bestpos[2]) * LAYER + bestpos[1]) * LAYER + bestpos[0] : -1;
        viaSum = zadd(viaSum, vu);
    }
    __syncwarp();
    if (lane < LAYER) {
        const int i = lane;
        int best = Z.map[idx_l], code = Z.prev[idx_l];
        bool changed = false;
        for (int lo = 0; lo <= i; ++lo)
            for (int up = i; up < LAYER; ++up) {
                const int c = cand[LAYER * LAYER + lo * LAYER + up];
                const int val = cand[lo * LAYER + up];
                if (c >= 0 && best > val) { best = val; code = c; changed = true; }
            }
        if (changed) { Z.map[idx_l] = best; Z.prev[idx_l] = code; }
    }
    __syncwarp();
}

// convert_routes (zshape_topology.hpp:249-290) of one (start, length | -1)
// pair straight into route words; returns a reference status on failure.
__device__ __forceinline__ int zemit(const Tables& T, const ZTrees& Z, int start, int len, int* r, int& out,
                                     long long cap) {
    const int n = Z.N;
    const int layer = start / (n * n) - 1;
    const int a = start / n % n, b = start % n;
    const bool ay = ((layer & 1) ^ T.DIR) != 0;
    const int x = ay ? a : b, y = ay ? b : a;
    if (layer < 0 || layer >= T.L || x >= T.X || y >= T.Y) return 3;
    const int pos0 = cell_index(T, layer, x, y);
    int pos1;
    if (len == -1) {
        if (layer + 1 >= T.L) return 3;
        pos1 = pos0 + T.XY;
    } else {
        const int end = start + len, ea = end / n % n, eb = end % n;
        const int ex = ay ? ea : eb, ey = ay ? eb : ea;
        if (ex >= T.X || ey >= T.Y) return 3;
        pos1 = cell_index(T, layer, ex, ey);
    }
    if (out + 1 < cap) { r[out++] = pos0; r[out++] = pos1; return 0; }
    return 1;
}

// Traceback (zshape.cuh:271-386) of one net on lane 0, converted into the
// net's route record.  Returns 0 or the reference's status (1 storage, 2 no
// finite route, 3 segment outside the grid).
__device__ __forceinline__ int ztrace(const Tables& T, const ZTrees& Z, int nb, int cnt, int* r, long long cap) {
    const int LAYER = Z.LAYER, N = Z.N, D = Z.D;
    int* map0 = Z.map;
    int* m5 = Z.map + 5 * Z.LNN;
    int out = 1, status = 0;
    auto emit = [&](int a, int b) { const int s = zemit(T, Z, a, b, r, out, cap); if (s) status = s; };
    int minTotal = kZInf;
    const int p0 = Z.pos[nb];
    for (int i = 0; i < LAYER; ++i) {
        const int idx = zidx(Z, i, p0 / N, p0 % N);
        if (map0[idx] < minTotal) { minTotal = map0[idx]; m5[p0] = i; }
    }
    if (minTotal == kZInf || minTotal < 0) { r[0] = 1; return 2; }
    for (int t = 0; t < cnt; ++t) {
        const int pt = Z.pos[nb + t], x = pt / N, y = pt % N, layer = m5[pt];
        const int idx = zidx(Z, layer, x, y);
        const int code = Z.prev[idx];
        const int minl = code / LAYER / LAYER / LAYER / LAYER, maxl = code / LAYER / LAYER / LAYER % LAYER;
        for (int i = minl; i < maxl; ++i) emit(zidx(Z, i, x, y), -1);
        int bestpos = code;
        for (int j = 0; j < 3; ++j) {
            const int c = Z.child[3 * (nb + t) + j];
            if (c == -1) break;
            const int child = Z.pos[nb + c];
            const int entrylayer = bestpos % LAYER, entry = zidx(Z, entrylayer, x, y);
            bestpos /= LAYER;
            const int last = Z.prev[(j + 1) * Z.LNN + entry];
            const int lastlayer = static_cast<int>(last / Z.NN);
            int lastx = last / N % N, lasty = last % N;
            if ((!(lastlayer & 1)) ^ D) { const int s = lastx; lastx = lasty; lasty = s; }
            if (lastx != x && lasty != y) {
                const int mid = Z.prev[(11 + j) * Z.LNN + entry];
                const int midlayer = static_cast<int>(mid / Z.NN);
                int midx = mid / N % N, midy = mid % N;
                if ((!(midlayer & 1)) ^ D) { const int s = midx; midx = midy; midy = s; }
                const int q1 = ((entrylayer & 1) ^ D) ? entry - y + midy : entry - x + midx;
                const int q3 = ((midlayer & 1) ^ D) ? mid - midy + lasty : mid - midx + lastx;
                const int q4 = ((lastlayer & 1) ^ D) ? last - lasty + midy : last - lastx + midx;
                if (entry != q1) emit(min(entry, q1), max(entry, q1) - min(entry, q1));
                if (q1 != mid)
                    for (int i = min(entrylayer, midlayer); i < max(entrylayer, midlayer); ++i) emit(zidx(Z, i, midx, midy), -1);
                if (mid != q3) emit(min(mid, q3), max(mid, q3) - min(mid, q3));
                if (q3 != q4) {
                    int tx = q3 / N % N, ty = q3 % N;
                    if ((!(static_cast<int>(q3 / Z.NN) & 1)) ^ D) { const int s = tx; tx = ty; ty = s; }
                    for (int i = min(midlayer, lastlayer); i < max(midlayer, lastlayer); ++i) emit(zidx(Z, i, tx, ty), -1);
                }
                if (q4 != last) emit(min(q4, last), max(q4, last) - min(q4, last));
            } else {
                emit(min(last, entry), max(last, entry) - min(last, entry));
            }
            m5[child] = lastlayer;
        }
    }
    r[0] = out;
    return status;
}

// Route net `id` with the whole CTA (thread t of nth); with `commit`, also its
// wire demand (warp 0).  `cand`: 2 * LAYER * LAYER ints of shared memory.
__device__ __forceinline__ void zshape_net(const Tables& T, const ZTrees& Z, const Plan& P, int id, int stamp,
                                           int t, int nth, bool commit, int* cand) {
    __shared__ int zstatus;
    const int lane = t;
    const int nb = Z.node_off[id], cnt = Z.node_off[id + 1] - nb;
    int* r = P.routes + P.route_off[id];
    const long long cap = P.route_off[id + 1] - P.route_off[id];
    if (cnt <= 0) {
        if (t == 0 && cap > 0) r[0] = 1;
        return;
    }
    // reset_nodes (zshape.cuh:392-404).
    for (int k = t; k < cnt * Z.LAYER; k += nth) {
        const int pt = Z.pos[nb + k / Z.LAYER];
        const int idx = zidx(Z, k % Z.LAYER, pt / Z.N, pt % Z.N);
        for (int plane = 0; plane < 4; ++plane) Z.map[plane * Z.LNN + idx] = kZInf;
    }
    __syncthreads();
    for (int v = cnt - 1; v >= 0; --v) {
        const int pt = Z.pos[nb + v], tox = pt / Z.N, toy = pt % Z.N;
        const int* ch = Z.child + 3 * (nb + v);
        for (int j = 1; j <= 3; ++j) {
            const int c = ch[j - 1];
            if (c == -1) continue;
            const int cp = Z.pos[nb + c];
            zedge(T, Z, j, cp / Z.N, cp % Z.N, tox, toy, lane, nth);
        }
        if (t < 32) znode_dp_warp(T, Z, tox, toy, Z.pin[nb + v], ch, lane, cand);
        __syncthreads();
    }
    if (t == 0) {
        zstatus = ztrace(T, Z, nb, cnt, r, cap);
        if (zstatus) set_error(T, zstatus == 1 ? kELimit : kEInval, id);
    }
    __syncthreads();
    const int status = zstatus;
    if (commit && !status && t < 32) commit_net_wires(T, P, id, stamp, 1, lane);
    __syncthreads();
}

// --- bounding-box batch refinement (zshape_topology.hpp:7-57) --------------
// Within one first-fit group, nets sorted by box area (descending, larger id
// first on ties) form greedy rounds of at most `max_batch` nets with pairwise
// disjoint boxes; this is first-fit colouring with box-intersection conflicts.
__device__ __forceinline__ bool boxes_meet(int4 a, int4 b) {
    // int4 = (minx, maxx, miny, maxy)
    return !(a.y < b.x || b.y < a.x || a.w < b.z || b.w < a.z);
}

}  // namespace grb
