// lshape.cuh -- L-shape pattern routing with layer assignment, one warp per net.
//
// Semantics are those of the reference's tree DP (lshape_thread.cuh:18-171,
// lshape_warp.cuh:8-247): per tree node a table dist[low][high] over layer
// ranges (via stack cost inside the range, INF where a pin's layer falls
// outside); children are merged into their parent in descending node order;
// an edge is a straight wire or an L with a via stack at the corner; strict '<'
// keeps the first minimum in the reference's loop order; the root takes the
// first minimal range; traceback and segment emission follow node order.
//
// B200 mapping: all cost gathers of a net (via stacks at nodes and corners,
// wire costs of both legs on every layer) are issued up front by the 32 lanes
// into a per-warp shared-memory arena, so a net pays one memory latency; the
// DP itself then runs from shared memory with lanes over layers.  The
// reference keeps 81 doubles per node in global scratch and gathers inside the
// DP loop.
#pragma once
#include "commit.cuh"
#include "common.cuh"

namespace grb {

__host__ __device__ __forceinline__ int tri_count(int L) { return L * (L + 1) / 2; }
__device__ __forceinline__ int tri(int L, int lo, int hi) { return lo * L - lo * (lo - 1) / 2 + (hi - lo); }

struct Arena {
    double* dist;          // [nmax][TT]
    double* w1;            // [nmax][L] first leg (or straight) wire cost
    double* w2;            // [nmax][L] second leg wire cost
    float* vA;             // [nmax][L] via cost at corner (x, py)
    float* vB;             // [nmax][L] via cost at corner (px, y)
    float* vN;             // [nmax][L] via cost at the node
    unsigned short* from;  // [nmax][TT] choice*L*L + curl*L + parl
    int* range;            // [nmax] chosen range lo*L+hi
    int* xy;               // [nmax] node coordinate x << 16 | y (grids are at most 8192 wide)
    int* lay;              // [nmax] node layer (L: Steiner point)
    int* dep;              // [nmax] node depth (root 0)
    // Per-lane scratch of a level pass: lane = slot * L + layer for up to
    // 32 / L nodes at once.
    double* cur;           // [32] best range through each layer (of the slot's node)
    double* diag;          // [32] best parent-layer cost
    int* cur_from;         // [32]
    int* pdiag;            // [32]
};

__host__ __device__ __forceinline__ size_t arena_bytes(int L, int nmax) {
    const size_t TT = tri_count(L);
    size_t b = 0;
    b += nmax * TT * 8 + 2 * size_t(nmax) * L * 8 + 3 * size_t(nmax) * L * 4;
    b = (b + 7) & ~size_t(7);
    b += 2 * 32 * 8;
    b += nmax * TT * 2;
    b = (b + 7) & ~size_t(7);
    b += nmax * 4 + 2 * 32 * 4 + 3 * size_t(nmax) * 4;
    return (b + 15) & ~size_t(15);
}

__device__ __forceinline__ Arena carve_arena(char* base, int L, int nmax) {
    const int TT = tri_count(L);
    Arena A;
    char* p = base;
    A.dist = reinterpret_cast<double*>(p); p += size_t(nmax) * TT * 8;
    A.w1 = reinterpret_cast<double*>(p); p += size_t(nmax) * L * 8;
    A.w2 = reinterpret_cast<double*>(p); p += size_t(nmax) * L * 8;
    A.vA = reinterpret_cast<float*>(p); p += size_t(nmax) * L * 4;
    A.vB = reinterpret_cast<float*>(p); p += size_t(nmax) * L * 4;
    A.vN = reinterpret_cast<float*>(p); p += size_t(nmax) * L * 4;
    p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t(7));
    A.cur = reinterpret_cast<double*>(p); p += 32 * 8;
    A.diag = reinterpret_cast<double*>(p); p += 32 * 8;
    A.from = reinterpret_cast<unsigned short*>(p); p += size_t(nmax) * TT * 2;
    p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 7) & ~uintptr_t(7));
    A.range = reinterpret_cast<int*>(p); p += nmax * 4;
    A.cur_from = reinterpret_cast<int*>(p); p += 32 * 4;
    A.pdiag = reinterpret_cast<int*>(p); p += 32 * 4;
    A.xy = reinterpret_cast<int*>(p); p += nmax * 4;
    A.lay = reinterpret_cast<int*>(p); p += nmax * 4;
    A.dep = reinterpret_cast<int*>(p);
    return A;
}

__device__ __forceinline__ double wire_cost(const Tables& T, int l, int xmin, int xmax, int ymin, int ymax) {
    // prefix_scan.cuh:10-40 (wire_segment_cost)
    return T.presum[cell_index(T, l, xmax, ymax)] - T.presum[cell_index(T, l, xmin, ymin)];
}

// Route one net.  All 32 lanes of the warp call this with the same id.
// Returns false (and records kELimit) if the net's route storage is too small.
// LC: the number of routing layers when known at compile time (the loops
// over layers then unroll into independent loads and predicated compares, in
// the same order), 0 for any layer count.
template <int LC>
__device__ __forceinline__ void lshape_net_l(const Tables& T, const Plan& P, int id, int stamp, const Arena& A,
                                             int lane, bool fuse_wires) {
    const int L = LC > 0 ? LC : T.L, Y = T.Y, XY = T.XY, TT = tri_count(L);
    constexpr int LL = LC > 0 ? LC : kMaxLayers;  // static bound of the layer loops
    const int off = P.node_off[id], N = P.node_off[id + 1] - off;
    const int* nd = P.nodes + off;
    const int* par = P.parents + off;

    // 0. Node coordinates, once per net (the divisions by the runtime grid
    // sizes are not repeated per layer and step).
    int dmax = 0;
    for (int q = lane; q < N; q += 32) {
        const int node = nd[q], l = node / XY, r = node - l * XY, x = r / Y;
        A.xy[q] = (x << 16) | (r - x * Y);
        A.lay[q] = l;
        int d = 0;
        for (int v = q; v > 0; v = par[v]) ++d;  // parents precede children
        A.dep[q] = d;
        dmax = max(dmax, d);
    }
    for (int s = 16; s; s >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, s));
    __syncwarp();
    // 1. Gather every cost the DP reads.  Each lane takes two (node, layer)
    // items per pass and issues all their loads before any arena store.
    for (int q0 = lane; q0 < N * L; q0 += 64) {
        float vn[2], va[2], vb[2];
        double w1[2], w2[2];
        int kind[2];  // 0: none, 1: node only, 2: straight edge, 3: L-shaped edge
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int q = q0 + 32 * u;
            kind[u] = 0;
            vn[u] = va[u] = vb[u] = 0.f;
            w1[u] = w2[u] = 0.0;
            if (q >= N * L) continue;
            const int i = q / L, l = q - i * L;
            const int x = A.xy[i] >> 16, y = A.xy[i] & 0xffff, r = x * Y + y;
            vn[u] = T.vcost[l * XY + r];
            kind[u] = 1;
            if (i > 0) {
                const int pxy = A.xy[par[i]], px = pxy >> 16, py = pxy & 0xffff;
                const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
                const bool ay = along_y(T, l);
                if (x == px || y == py) {
                    const bool valid = ay ? (x == px) : (y == py);
                    w1[u] = valid ? wire_cost(T, l, minx, maxx, miny, maxy) : 0.0;
                    kind[u] = 2;
                } else {
                    w1[u] = ay ? wire_cost(T, l, x, x, miny, maxy) : wire_cost(T, l, minx, maxx, y, y);
                    w2[u] = ay ? wire_cost(T, l, px, px, miny, maxy) : wire_cost(T, l, minx, maxx, py, py);
                    va[u] = T.vcost[cell_index(T, l, x, py)];
                    vb[u] = T.vcost[cell_index(T, l, px, y)];
                    kind[u] = 3;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int q = q0 + 32 * u;
            if (kind[u] >= 1) A.vN[q] = vn[u];
            if (kind[u] >= 2) A.w1[q] = w1[u];
            if (kind[u] == 3) {
                A.w2[q] = w2[u];
                A.vA[q] = va[u];
                A.vB[q] = vb[u];
            }
        }
    }
    __syncwarp();
    // 2. Via stacks at every node (lshape_thread.cuh:40-50).
    for (int q = lane; q < N * L; q += 32) {
        const int i = q / L, lo = q - i * L;
        const int fixed = A.lay[i];
        double acc = 0;
#pragma unroll
        for (int hi = 0; hi < LL; ++hi) {
            if (hi < lo || hi >= L) continue;
            if (hi > lo) acc = acc + static_cast<double>(A.vN[i * L + hi - 1]);
            A.dist[i * TT + tri(L, lo, hi)] = (fixed < L && (lo > fixed || hi < fixed)) ? kInf : acc;
        }
    }
    __syncwarp();
    // 3. Children into parents (lshape_thread.cuh:51-115), one depth at a
    // time from the deepest: the nodes of a depth have complete tables, so
    // up to 32 / L of them are processed at once (lane = slot * L + layer);
    // then every node of the depth, in descending node order, adds its table
    // into its parent.  A parent receives its children (all one depth below
    // it) in descending order, exactly the sequential loop's additions.
    const int S = max(1, 32 / L);
    const int slot = lane / L, sl = lane - slot * L;
    for (int d = dmax; d >= 1; --d) {
        for (int base = 0; base < N; base += 32) {
            const int q = base + lane;
            unsigned at = __ballot_sync(0xffffffffu, q < N && A.dep[q] == d);
            while (at) {
                // The next S nodes of this depth in this window.
                int mine = -1;
                {
                    unsigned m = at;
                    for (int k = 0; k < S && m; ++k) {
                        const int b = __ffs(m) - 1;
                        m &= m - 1;
                        if (k == slot) mine = base + b;
                    }
                    at = m;
                }
                const bool act = slot < S && mine >= 0;
                const int i = mine;
                if (act) {
                    const double* di = A.dist + i * TT;
                    const int l = sl;
                    double best = kInf;
                    int bf = 0;
#pragma unroll
                    for (int lo = 0; lo < LL; ++lo)
#pragma unroll
                        for (int hi = lo; hi < LL; ++hi) {
                            if (lo > l || hi < l || hi >= L) continue;
                            const double v = di[tri(L, lo, hi)];
                            if (v < best) { best = v; bf = lo * L + hi; }
                        }
                    A.cur[lane] = best;
                    A.cur_from[lane] = bf;
                }
                __syncwarp();
                if (act) {
                    const int pl = sl, p = par[i], s0 = slot * L;
                    const int x = A.xy[i] >> 16, y = A.xy[i] & 0xffff;
                    const int px = A.xy[p] >> 16, py = A.xy[p] & 0xffff;
                    double best = kInf;
                    int pb = 0;
                    if (x == px || y == py) {
                        const bool valid = along_y(T, pl) ? (x == px) : (y == py);
                        if (valid) {
                            best = A.cur[s0 + pl] + A.w1[i * L + pl];
                            pb = A.cur_from[s0 + pl] * L * L + pl * L + pl;
                        }
                    } else {
#pragma unroll
                        for (int cl = 0; cl < LL; ++cl) {
                            if (((cl ^ pl) & 1) == 0 || cl >= L) continue;  // the other parity, ascending
                            const double cost = A.cur[s0 + cl] + A.w1[i * L + cl];
                            double cost2 = 0;
                            const float* v = along_y(T, cl) ? A.vA + i * L : A.vB + i * L;
                            const int a = min(cl, pl), b = max(cl, pl);
#pragma unroll
                            for (int l = 0; l < LL; ++l)
                                if (l > a && l < b) cost2 += static_cast<double>(v[l]);
                            cost2 += A.w2[i * L + pl];
                            if (cost + cost2 < best) {
                                best = cost + cost2;
                                pb = A.cur_from[s0 + cl] * L * L + cl * L + pl;
                            }
                        }
                    }
                    A.diag[lane] = best;
                    A.pdiag[lane] = pb;
                }
                __syncwarp();
                if (act) {
                    // The node's contribution to its parent replaces its own
                    // table (read above, not needed again).
                    const int lo = sl, s0 = slot * L;
                    double c = A.diag[s0 + lo];
                    int path = A.pdiag[s0 + lo];
#pragma unroll
                    for (int hi = 0; hi < LL; ++hi) {
                        if (hi < lo || hi >= L) continue;
                        if (hi > lo && !(c <= A.diag[s0 + hi])) { c = A.diag[s0 + hi]; path = A.pdiag[s0 + hi]; }
                        const int t = tri(L, lo, hi);
                        A.dist[i * TT + t] = c;
                        A.from[i * TT + t] = static_cast<unsigned short>(path);
                    }
                }
                __syncwarp();
            }
        }
        for (int i = N - 1; i >= 1; --i) {
            if (A.dep[i] != d) continue;
            const int p = par[i];
            for (int t = lane; t < TT; t += 32) A.dist[p * TT + t] += A.dist[i * TT + t];
            __syncwarp();
        }
    }
    // 4. Root range (lshape_thread.cuh:117-120): the first minimum in loop
    // order (lo, then hi), i.e. the smallest triangular index among equal
    // values -- a warp argmin; then the traceback one depth at a time.
    {
        double bv = __longlong_as_double(0x7ff0000000000000ll);  // +infinity: every finite entry is below it
        int bt = 1 << 30;
        for (int t = lane; t < TT; t += 32) {
            const double v = A.dist[t];
            if (v < bv) { bv = v; bt = t; }
        }
        for (int s = 16; s; s >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, s);
            const int ot = __shfl_xor_sync(0xffffffffu, bt, s);
            if (ov < bv || (ov == bv && ot < bt)) { bv = ov; bt = ot; }
        }
        if (lane == 0) {
            if (bt >= TT) bt = 0;  // no entry below infinity: the sequential loop keeps index 0
            int lo = 0;
            while (lo + 1 < L && tri(L, lo + 1, lo + 1) <= bt) ++lo;
            A.range[0] = lo * L + (lo + bt - tri(L, lo, lo));
            if (!(bv < kInf)) set_error(T, kEInval, id);
        }
    }
    __syncwarp();
    for (int d = 1; d <= dmax; ++d) {
        for (int i = lane; i < N; i += 32) {
            if (i == 0 || A.dep[i] != d) continue;
            const int pr = A.range[par[i]];
            A.range[i] = A.from[i * TT + tri(L, pr / L, pr % L)] / (L * L);
        }
        __syncwarp();
    }
    // 5. Segment emission in node order (lshape_warp.cuh:215-240).
    int* out = P.routes + P.route_off[id];
    const long long cap = P.route_off[id + 1] - P.route_off[id];
    int next = 1;
    for (int b0 = 0; b0 < N; b0 += 32) {
        const int i = b0 + lane;
        int words = 0, x = 0, y = 0, px = 0, py = 0, cl = 0, pl = 0, minl = 0, maxl = 0;
        if (i < N) {
            x = A.xy[i] >> 16; y = A.xy[i] & 0xffff;
            minl = A.range[i] / L; maxl = A.range[i] % L;
            words = minl < maxl ? 2 : 0;
            if (i) {
                px = A.xy[par[i]] >> 16; py = A.xy[par[i]] & 0xffff;
                const int pr = A.range[par[i]];
                const int f = A.from[i * TT + tri(L, pr / L, pr % L)];
                cl = f / L % L; pl = f % L;
                words += (x == px || y == py) ? 2 : 6;
            }
        }
        int prefix = words;
        for (int s = 1; s < 32; s <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, prefix, s);
            if (lane >= s) prefix += o;
        }
        const int total = __shfl_sync(0xffffffffu, prefix, 31);
        if (next + total > cap) {
            if (lane == 0) set_error(T, kELimit, id);
            return;
        }
        if (i < N) {
            int* w = out + next + prefix - words;
            if (minl < maxl) { *w++ = cell_index(T, minl, x, y); *w++ = cell_index(T, maxl, x, y); }
            if (i) {
                if (x == px || y == py) {
                    *w++ = cell_index(T, cl, min(x, px), min(y, py));
                    *w++ = cell_index(T, cl, max(x, px), max(y, py));
                } else if (along_y(T, cl)) {
                    *w++ = cell_index(T, cl, x, y);   *w++ = cell_index(T, cl, x, py);
                    *w++ = cell_index(T, cl, x, py);  *w++ = cell_index(T, pl, x, py);
                    *w++ = cell_index(T, pl, x, py);  *w++ = cell_index(T, pl, px, py);
                } else {
                    *w++ = cell_index(T, cl, x, y);   *w++ = cell_index(T, cl, px, y);
                    *w++ = cell_index(T, cl, px, y);  *w++ = cell_index(T, pl, px, y);
                    *w++ = cell_index(T, pl, px, y);  *w++ = cell_index(T, pl, px, py);
                }
            }
        }
        next += total;
    }
    if (lane == 0) out[0] = next;
    __syncwarp();
    if (fuse_wires) commit_net_wires(T, P, id, stamp, 1, lane);
}

// Route one net: the layer loops unrolled for the 9 routing layers of the
// reference's 10-layer designs, generic otherwise.
__device__ __forceinline__ void lshape_net(const Tables& T, const Plan& P, int id, int stamp, const Arena& A,
                                           int lane, bool fuse_wires) {
    if (T.L == 9) lshape_net_l<9>(T, P, id, stamp, A, lane, fuse_wires);
    else lshape_net_l<0>(T, P, id, stamp, A, lane, fuse_wires);
}

// Nets of one or two tree nodes, one net per lane: the lanes of a warp route
// up to 32 such nets at once (most nets of a design), where lshape_net would
// spend a whole warp, mostly idle, on each.  Same arithmetic, comparisons,
// tie-breaks and emission order as lshape_net on the same net, so the routes
// are identical.  Scratch: lane-interleaved per-warp shared memory of
// pair_scratch_bytes().  id < 0: the lane has no net.
constexpr int kPairD = 3 * kMaxLayers;  // doubles per lane: cur, w1, w2 (then diag)
constexpr int kPairF = 3 * kMaxLayers;  // 4-byte words per lane: vA (then root vN), vB, vN (then choices)
constexpr int kPairH = kMaxLayers;      // shorts per lane: best range through each layer
__host__ __device__ __forceinline__ size_t pair_scratch_bytes() {
    return size_t(32) * (kPairD * 8 + kPairF * 4 + kPairH * 2);
}

template <int LC>
__device__ __forceinline__ void lshape_net_pair_l(const Tables& T, const Plan& P, int id, int stamp, char* scratch,
                                                  int lane, bool commit) {
    if (id < 0) return;
    double* sd = reinterpret_cast<double*>(scratch);
    float* sf = reinterpret_cast<float*>(scratch + size_t(32) * kPairD * 8);
    int* si = reinterpret_cast<int*>(sf);
    unsigned short* sh = reinterpret_cast<unsigned short*>(scratch + size_t(32) * (kPairD * 8 + kPairF * 4));
    auto cur = [&](int l) -> double& { return sd[l * 32 + lane]; };
    auto w1 = [&](int l) -> double& { return sd[(kMaxLayers + l) * 32 + lane]; };
    auto w2 = [&](int l) -> double& { return sd[(2 * kMaxLayers + l) * 32 + lane]; };    // then diag
    auto vA = [&](int l) -> float& { return sf[l * 32 + lane]; };                           // then root vN
    auto vB = [&](int l) -> float& { return sf[(kMaxLayers + l) * 32 + lane]; };
    auto vN = [&](int l) -> float& { return sf[(2 * kMaxLayers + l) * 32 + lane]; };
    auto pdiag = [&](int l) -> int& { return si[(2 * kMaxLayers + l) * 32 + lane]; };       // after vN
    auto cfrom = [&](int l) -> unsigned short& { return sh[l * 32 + lane]; };
    const int L = LC > 0 ? LC : T.L, Y = T.Y, XY = T.XY;
    const int off = P.node_off[id], N = P.node_off[id + 1] - off;
    const int n0 = P.nodes[off], r0 = n0 % XY, x0 = r0 / Y, y0 = r0 - x0 * Y, fix0 = n0 / XY;
    int x1 = 0, y1 = 0;
    bool straight = false;
    if (N == 2) {
        const int n1 = P.nodes[off + 1], r1 = n1 % XY, fix1 = n1 / XY;
        x1 = r1 / Y;
        y1 = r1 - x1 * Y;
        straight = x1 == x0 || y1 == y0;
        const int minx = min(x1, x0), maxx = max(x1, x0), miny = min(y1, y0), maxy = max(y1, y0);
        // Step 1 for node 1 (the child), kHalfLayers layers at a time: every
        // load of a group is issued before its stores.
        constexpr int kHalfLayers = kMaxLayers / 2;
#pragma unroll
        for (int l0 = 0; l0 < kMaxLayers; l0 += kHalfLayers) {
            float vn[kHalfLayers], va[kHalfLayers], vb[kHalfLayers];
            double a[kHalfLayers], b[kHalfLayers];
#pragma unroll
            for (int u = 0; u < kHalfLayers; ++u) {
                const int l = l0 + u;
                vn[u] = va[u] = vb[u] = 0.f;
                a[u] = b[u] = 0.0;
                if (l >= L) continue;
                const bool ay = along_y(T, l);
                vn[u] = T.vcost[l * XY + r1];
                if (straight) {
                    const bool valid = ay ? (x1 == x0) : (y1 == y0);
                    a[u] = valid ? wire_cost(T, l, minx, maxx, miny, maxy) : 0.0;
                } else {
                    a[u] = ay ? wire_cost(T, l, x1, x1, miny, maxy) : wire_cost(T, l, minx, maxx, y1, y1);
                    b[u] = ay ? wire_cost(T, l, x0, x0, miny, maxy) : wire_cost(T, l, minx, maxx, y0, y0);
                    va[u] = T.vcost[cell_index(T, l, x1, y0)];
                    vb[u] = T.vcost[cell_index(T, l, x0, y1)];
                }
            }
#pragma unroll
            for (int u = 0; u < kHalfLayers; ++u) {
                const int l = l0 + u;
                if (l >= L) continue;
                vN(l) = vn[u];
                w1(l) = a[u];
                w2(l) = b[u];
                vA(l) = va[u];
                vB(l) = vb[u];
            }
        }
        // Steps 2 and 3a: the child's via stacks, and its best range through
        // each layer, first minimum in (lo, hi) order.
#pragma unroll
        for (int l = 0; l < L; ++l) {
            cur(l) = kInf;
            cfrom(l) = 0;
        }
#pragma unroll
        for (int lo = 0; lo < L; ++lo) {
            double acc = 0;
#pragma unroll
            for (int hi = lo; hi < L; ++hi) {
                if (hi > lo) acc = acc + static_cast<double>(vN(hi - 1));
                const double v = (fix1 < L && (lo > fix1 || hi < fix1)) ? kInf : acc;
#pragma unroll
                for (int l = lo; l <= hi; ++l)
                    if (v < cur(l)) {
                        cur(l) = v;
                        cfrom(l) = static_cast<unsigned short>(lo * L + hi);
                    }
            }
        }
        // Step 3b: best cost of reaching the parent on each layer.
#pragma unroll
        for (int pl = 0; pl < L; ++pl) {
            double best = kInf;
            int pb = 0;
            if (straight) {
                const bool valid = along_y(T, pl) ? (x1 == x0) : (y1 == y0);
                if (valid) {
                    best = cur(pl) + w1(pl);
                    pb = cfrom(pl) * L * L + pl * L + pl;
                }
            } else {
#pragma unroll
                for (int cl = (pl & 1) ^ 1; cl < L; cl += 2) {
                    const double cost = cur(cl) + w1(cl);
                    double cost2 = 0;
                    const bool ay = along_y(T, cl);
#pragma unroll
                    for (int l = min(cl, pl) + 1; l < max(cl, pl); ++l)
                        cost2 += static_cast<double>(ay ? vA(l) : vB(l));
                    cost2 += w2(pl);
                    if (cost + cost2 < best) {
                        best = cost + cost2;
                        pb = cfrom(cl) * L * L + cl * L + pl;
                    }
                }
            }
            w2(pl) = best;   // w2(pl) is not read again
            pdiag(pl) = pb;  // vN of the child is not read again
        }
    }
    // The root's via-cost column (vA of the child is not read again).
    {
        float v[kMaxLayers];
#pragma unroll
        for (int l = 0; l < kMaxLayers; ++l) v[l] = l < L ? T.vcost[l * XY + r0] : 0.f;
#pragma unroll
        for (int l = 0; l < kMaxLayers; ++l)
            if (l < L) vA(l) = v[l];
    }
    // Steps 2, 3c, 3d and 4 for the root: its via stacks plus, for a child,
    // the range minimum of the diagonal; the first minimal range.
    int choice = 0, bestpath = 0;
    {
        double best = 0;
#pragma unroll
        for (int lo = 0; lo < L; ++lo) {
            double acc = 0, c = 0;
            int path = 0;
            if (N == 2) {
                c = w2(lo);
                path = pdiag(lo);
            }
#pragma unroll
            for (int hi = lo; hi < L; ++hi) {
                if (hi > lo) acc = acc + static_cast<double>(vA(hi - 1));
                double v = (fix0 < L && (lo > fix0 || hi < fix0)) ? kInf : acc;
                if (N == 2) {
                    if (hi > lo && !(c <= w2(hi))) {
                        c = w2(hi);
                        path = pdiag(hi);
                    }
                    v += c;
                }
                if ((lo == 0 && hi == 0) || v < best) {
                    best = v;
                    choice = lo * L + hi;
                    bestpath = path;
                }
            }
        }
        if (!(best < kInf)) set_error(T, kEInval, id);
    }
    // Step 5: segments in node order.
    int* out = P.routes + P.route_off[id];
    const long long cap = P.route_off[id + 1] - P.route_off[id];
    const int minl0 = choice / L, maxl0 = choice % L;
    int words = minl0 < maxl0 ? 2 : 0;
    int minl1 = 0, maxl1 = 0, cl = 0, pl = 0;
    if (N == 2) {
        const int r1 = bestpath / (L * L);
        minl1 = r1 / L;
        maxl1 = r1 % L;
        cl = bestpath / L % L;
        pl = bestpath % L;
        words += (minl1 < maxl1 ? 2 : 0) + (straight ? 2 : 6);
    }
    if (1 + words > cap) {
        set_error(T, kELimit, id);
        return;
    }
    int* w = out + 1;
    if (minl0 < maxl0) { *w++ = cell_index(T, minl0, x0, y0); *w++ = cell_index(T, maxl0, x0, y0); }
    if (N == 2) {
        if (minl1 < maxl1) { *w++ = cell_index(T, minl1, x1, y1); *w++ = cell_index(T, maxl1, x1, y1); }
        if (straight) {
            *w++ = cell_index(T, cl, min(x1, x0), min(y1, y0));
            *w++ = cell_index(T, cl, max(x1, x0), max(y1, y0));
        } else if (along_y(T, cl)) {
            *w++ = cell_index(T, cl, x1, y1);   *w++ = cell_index(T, cl, x1, y0);
            *w++ = cell_index(T, cl, x1, y0);   *w++ = cell_index(T, pl, x1, y0);
            *w++ = cell_index(T, pl, x1, y0);   *w++ = cell_index(T, pl, x0, y0);
        } else {
            *w++ = cell_index(T, cl, x1, y1);   *w++ = cell_index(T, cl, x0, y1);
            *w++ = cell_index(T, cl, x0, y1);   *w++ = cell_index(T, pl, x0, y1);
            *w++ = cell_index(T, pl, x0, y1);   *w++ = cell_index(T, pl, x0, y0);
        }
    }
    out[0] = 1 + words;
    if (commit) commit_thread_wires(T, P, id, stamp, 1);
}

// One or two tree nodes per lane: unrolled for 9 routing layers, generic
// otherwise.
__device__ __forceinline__ void lshape_net_pair(const Tables& T, const Plan& P, int id, int stamp, char* scratch,
                                                int lane, bool commit) {
    if (T.L == 9) lshape_net_pair_l<9>(T, P, id, stamp, scratch, lane, commit);
    else lshape_net_pair_l<0>(T, P, id, stamp, scratch, lane, commit);
}

}  // namespace grb
