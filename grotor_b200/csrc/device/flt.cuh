// flt.cuh -- FLT stage: mid-edge layer-change tables, DAG solve and trace.
//
// Semantics of the reference's FLT execution (flt_cost.cuh:25-130,
// flt_block.cuh:6-355).  Each net carries a DAG whose nodes are 3-D grid
// points (layer 9 = no pin layer) and whose edges connect a child node to one
// of its parents' child slots; alternative nodes compete for a slot.  Solve
// runs from the deepest level up: a node combines, per layer, the cheapest
// candidate of every child slot plus its via stack, then offers every parent
// slot a packed (fp32 cost, node*100 + choice) key per target layer, kept by
// a 64-bit atomicMin.  Trace runs from the root down and emits the chosen
// wires (straight, or split at the best sampled mid-edge layer change) and
// each node's via stack.
//
// B200 form: the layer-change tables of all the batch's edges are one
// grid-wide pass, a thread per (edge, from-layer, to-layer) entry (the
// reference launches a thread per (edge, from-layer)); then one warp per net
// (the reference uses a 128-thread CTA); lanes take the nodes of one depth
// level, __syncwarp separates levels; the packed keys live in a per-stage
// workspace in HBM (mostly L2-resident per batch).
// Node numbering is net-local: candidates for a slot always belong to one
// net, so the batch-global numbering of the reference orders them the same.
// Segments are appended in level order, ascending node index within a level,
// each node's wires before its via stack (the reference appends with atomics,
// so only its segment multiset is defined).
#pragma once
#include "commit.cuh"
#include "common.cuh"

namespace grb {

constexpr int kFltLayers = 10;                                  // MAX_LAYER, flt_cost.cuh:14
constexpr unsigned long long kFltInit = 7208259049189261824ull; // init_cost_with_road, flt_cost.cuh:48
constexpr int kFltStraight = 82;                                // flt_block.cuh:109
constexpr int kFltMaxChildren = 6;                              // flt_block.cuh:31-32

struct Flt {
    // per net id
    const int* node_off;     // [n+1] global node index of the net's node 0
    const int* edge_off;     // [n+1] global edge index of the net's edge 0
    const int* lvl_off;      // [n+1] into level: the net's depth levels
    const long long* route2_off;  // [n+1] phase-two route words
    // per depth level: first position in `order` (net-local), plus one end
    // entry per net at lvl_off[id+1]-1 ... stored as level[lvl_off[id] + d]
    const int* level;        // [sum over nets of depths+1]
    // per node (global index)
    const int* coord;        // l*X*Y + x*Y + y
    const int* children;     // child slots
    const int* child_off;    // global exclusive prefix of children
    const int* pend;         // net-local cumulative parent-edge count
    const int* order;        // net-local node indices by (depth, index)
    // per edge (global index)
    const int* eparent;      // net-local parent node
    const int* eslot;        // source slot: child node (net-local) * 10 + slot index at the parent
    // workspace
    double* costs;                 // [nodes*10]
    unsigned long long* packed;    // [children*10]
    unsigned long long* best;      // [children*10]
    int* lo;                       // [nodes] chosen layer (1-based), -1 unused
    double* ce;                    // [edges*81] layer-change cost
    int* bc;                       // [edges*81] layer-change position
    int* routes2;
    // per plan position: first edge slot (exclusive prefix of the plan's
    // edges, [plan+1]); per edge slot: its plan position
    const int* eprefix;
    const int* emap;
    // per plan position, batch by batch: the batch's positions with its wide
    // nets (a DAG level wider than a warp) first; per batch: its wide nets
    const int* border;
    const int* nwide;
};

__device__ __forceinline__ double flt_wire(const Tables& T, int l, int xmin, int xmax, int ymin, int ymax) {
    // prefix_scan.cuh:10-40 (wire_segment_cost)
    return T.presum[cell_index(T, l, xmax, ymax)] - T.presum[cell_index(T, l, xmin, ymin)];
}

// flt_cost.cuh:25-46.
__device__ __forceinline__ unsigned long long flt_pack(float cost, int id) {
    int i = __float_as_int(cost);
    i = i >= 0 ? i : i ^ 0x7FFFFFFF;
    return (static_cast<unsigned long long>(static_cast<unsigned>(i)) << 32) | static_cast<unsigned>(id);
}
__device__ __forceinline__ double flt_cost(unsigned long long p) {
    int i = static_cast<int>(p >> 32);
    i = i >= 0 ? i : i ^ 0x7FFFFFFF;
    return static_cast<double>(__int_as_float(i));
}

// precompute_cost_edge (flt_cost.cuh:50-130) for every (from-layer,
// to-layer) entry of global edge `e`, one warp.  Entries the solve never
// reads -- an edge with a bend or of Manhattan length <= 4 (only straight
// wires are offered there), a from-layer across the edge's direction, a
// to-layer of the other parity -- are INF with position -1.  Otherwise the
// entry is the cheapest layer change over the sampled positions (every
// dd-th position strictly inside the edge, dd = distance / min(distance,
// 20)): the via stack between the layers there plus the wire from each end
// to it on its layer, the via costs added from the lower layer up and the two
// wires summed before they are added, the first minimum in increasing
// position kept.  Lanes take the positions (32 at a time) and evaluate every
// entry there; the first minimum comes from a warp reduction of (cost,
// position) pairs.
__device__ __forceinline__ void flt_edge_warp(const Tables& T, const Flt& F, int nb, int e, int lane) {
    const int to = nb + F.eparent[e], from = nb + F.eslot[e] / 10;
    const int ct = F.coord[to], cf = F.coord[from];
    const int tox = ct / T.Y % T.X, toy = ct % T.Y, fromx = cf / T.Y % T.X, fromy = cf % T.Y;
    double* ce = F.ce + size_t(e) * 81;
    int* bc = F.bc + size_t(e) * 81;
    for (int k = lane; k < 81; k += 32) { ce[k] = kInf; bc[k] = -1; }
    const int distance = abs(tox - fromx) + abs(toy - fromy);
    const bool vertical = fromx == tox;
    if (distance <= 4 || (!vertical && fromy != toy)) return;
    __syncwarp();  // the fill above comes before the entries below
    const int dd = distance / min(distance, 20);
    const int start = vertical ? min(fromy, toy) : min(fromx, tox);
    const int end = vertical ? max(fromy, toy) : max(fromx, tox);
    const int ns = start + dd < end ? (end - 1 - (start + dd)) / dd + 1 : 0;  // sampled positions
    // Layers of the edge's direction (the only from- and to-layers with
    // finite entries): l0, l0 + 2, ...
    const int l0 = (vertical ? (T.DIR ^ 1) : T.DIR) & 1;
    constexpr int KV = (kFltLayers + 1) / 2;
    for (int fi = 0; fi < KV; ++fi) {
        const int fl = l0 + 2 * fi;
        if (fl >= 9 || fl >= T.L) break;
        double bv[KV];
        int bp[KV];
#pragma unroll
        for (int ti = 0; ti < KV; ++ti) { bv[ti] = kInf; bp[ti] = -1; }
        const double pF = T.presum[cell_index(T, fl, fromx, fromy)];
        for (int base = 0; base < ns; base += 32) {
            const int s = base + lane;
            if (s < ns) {
                const int sp = start + dd + s * dd;
                const int sx = vertical ? fromx : sp, sy = vertical ? sp : fromy;
                float vc[kFltLayers];
#pragma unroll
                for (int ll = 0; ll < kFltLayers - 1; ++ll) vc[ll] = ll < T.L ? T.vcost[cell_index(T, ll, sx, sy)] : 0.f;
                const double pf = T.presum[cell_index(T, fl, sx, sy)];
                const double wf = vertical ? (sy > fromy ? pf - pF : pF - pf) : (sx > fromx ? pf - pF : pF - pf);
#pragma unroll
                for (int ti = 0; ti < KV; ++ti) {
                    const int tl = l0 + 2 * ti;
                    if (tl >= 9 || tl >= T.L) continue;
                    const double pT = T.presum[cell_index(T, tl, tox, toy)];
                    const double pt = T.presum[cell_index(T, tl, vertical ? tox : sp, vertical ? sp : toy)];
                    const double wt = vertical ? (sy > toy ? pt - pT : pT - pt) : (sx > tox ? pt - pT : pT - pt);
                    const int lo = min(fl, tl), hi = max(fl, tl);
                    double via = 0;
#pragma unroll
                    for (int ll = 0; ll < kFltLayers - 1; ++ll)
                        if (ll >= lo && ll < hi) via += vc[ll];  // in increasing order, as the reference adds
                    double c = via;
                    c += (wf + wt);
                    if (c < bv[ti]) { bv[ti] = c; bp[ti] = sp; }
                }
            }
        }
#pragma unroll
        for (int ti = 0; ti < KV; ++ti) {
            const int tl = l0 + 2 * ti;
            if (tl >= 9 || tl >= T.L) continue;
            double v = bv[ti];
            int p = bp[ti];
            for (int o = 16; o; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, v, o);
                const int op = __shfl_down_sync(0xffffffffu, p, o);
                if (op >= 0 && (p < 0 || ov < v || (ov == v && op < p))) { v = ov; p = op; }
            }
            if (lane == 0 && p >= 0) { ce[fl * 9 + tl] = v; bc[fl * 9 + tl] = p; }
        }
    }
}

// The layer-change tables of every edge of batch b, one warp per edge over
// warps w, w + nw, ...: the reference's precompute_cost_edge launch over the
// batch's edges (flt.cuh:152).  Edge slot s of the plan belongs to plan
// position emap[s]; eprefix[k] is the first slot of position k.
__device__ __forceinline__ void flt_edges_batch(const Tables& T, const Flt& F, const Plan& P, int b, long long w,
                                                long long nw, int lane) {
    const int lo = P.batch_off[b], hi = P.batch_off[b + 1];
    const long long s0 = F.eprefix[lo], items = static_cast<long long>(F.eprefix[hi]) - s0;
    for (long long q = w; q < items; q += nw) {
        const int s = static_cast<int>(s0 + q);
        const int k = F.emap[s];
        const int id = P.ids[k];
        flt_edge_warp(T, F, F.node_off[id], F.edge_off[id] + (s - F.eprefix[k]), lane);
    }
}

// solve_flt_node (flt_block.cuh:6-142) for net-local node `i`.  The node's
// inputs -- its children's candidate keys and the via costs of its column --
// are loaded once, and its range costs and choices are kept in registers and
// thread-local arrays until the end (in HBM they would cost a round trip per
// read after a write); the loops and comparisons are the reference's.
__device__ __forceinline__ void flt_solve_node(const Tables& T, const Flt& F, int nb, int eb, int i) {
    const int g = nb + i;
    const int c0 = F.coord[g];
    const int flow = 1 + c0 / T.XY, x = c0 / T.Y % T.X, y = c0 % T.Y;
    const int fhigh = flow == kFltLayers ? 0 : flow;
    const int nc = F.children[g];
    unsigned long long* cbp = F.best + size_t(F.child_off[g]) * kFltLayers;
    const unsigned long long* cpk = F.packed + size_t(F.child_off[g]) * kFltLayers;
    double* cst_g = F.costs + size_t(g) * kFltLayers;
    unsigned long long pk[kFltMaxChildren][kFltLayers];  // children's keys
    for (int c = 0; c < nc; ++c) {
        unsigned long long v[kFltLayers];
#pragma unroll
        for (int li = 0; li < kFltLayers; ++li) v[li] = cpk[c * kFltLayers + li];
#pragma unroll
        for (int li = 0; li < kFltLayers; ++li) pk[c][li] = v[li];
    }
    float vc[kFltLayers];  // via cost of routing layer li - 2 at the node
#pragma unroll
    for (int li = 2; li < kFltLayers; ++li) vc[li] = li - 2 < T.L ? T.vcost[cell_index(T, li - 2, x, y)] : 0.f;
    double cst[kFltLayers];
#pragma unroll
    for (int li = 0; li < kFltLayers; ++li) cst[li] = kInf;  // as flt_net left them
    unsigned long long chosen[kFltMaxChildren][kFltLayers];  // chosen child candidate per range top
    unsigned written = 0;                                    // range tops whose choices were set
    double mcc[kFltMaxChildren];
    unsigned long long bp[kFltMaxChildren];
    for (int c = 0; c < kFltMaxChildren; ++c) bp[c] = 0;
    for (int low = 1; low <= flow; ++low) {
        for (int c = 0; c < nc; ++c) mcc[c] = kInf;
        double via = 0;
#pragma unroll
        for (int li = 1; li < kFltLayers; ++li) {
            if (li < low || li >= T.L + 1) continue;
            if (li > low) via += vc[li];
            for (int c = 0; c < nc; ++c) {
                const unsigned long long pv = pk[c][li];
                const double cc = flt_cost(pv);
                if (cc < mcc[c]) { mcc[c] = cc; bp[c] = static_cast<unsigned long long>(static_cast<unsigned>(pv)) * kFltLayers + li; }
            }
            if (li >= fhigh) {
                double cost = via;
                for (int c = 0; c < nc; ++c) cost += mcc[c];
                if (cost < kInf && cost < cst[li]) {
                    cst[li] = cost;
                    for (int c = 0; c < nc; ++c) chosen[c][li] = bp[c];
                    written |= 1u << li;
                }
            }
        }
#pragma unroll
        for (int li = kFltLayers - 2; li >= 1; --li) {
            if (li < low || li > T.L - 1) continue;
            if (cst[li + 1] < cst[li]) {
                cst[li] = cst[li + 1];
                for (int c = 0; c < nc; ++c) chosen[c][li] = chosen[c][li + 1];
                written |= 1u << li;
            }
        }
    }
#pragma unroll
    for (int li = 0; li < kFltLayers; ++li) cst_g[li] = cst[li];
    for (int c = 0; c < nc; ++c)
#pragma unroll
        for (int li = 0; li < kFltLayers; ++li)
            if (written >> li & 1u) cbp[c * kFltLayers + li] = chosen[c][li];
    const int pb = i ? F.pend[g - 1] : 0, pe = F.pend[g];
    for (int e = eb + pb; e < eb + pe; ++e) {
        const int par = nb + F.eparent[e], slot = F.eslot[e] % 10;
        unsigned long long* ppk = F.packed + size_t(F.child_off[par]) * kFltLayers + slot * kFltLayers;
        const int cp = F.coord[par], px = cp / T.Y % T.X, py = cp % T.Y;
        const int minx = min(x, px), maxx = max(x, px), miny = min(y, py), maxy = max(y, py);
        const bool far = abs(x - px) + abs(y - py) > 4;
        unsigned long long cache[kFltLayers];
        for (int t = 0; t < kFltLayers; ++t) cache[t] = kFltInit;
#pragma unroll
        for (int layer = 1; layer < kFltLayers; ++layer) {
            const bool ay = ((layer & 1) ^ T.DIR) == 1;  // 1-based layer index
            if (ay && y != py) continue;
            if (!ay && x != px) continue;
            const double cb = cst[layer];
            for (int tl = 1 + (1 - layer % 2); tl < kFltLayers; tl += 2) {
                double c2;
                int choice = kFltStraight;
                if (tl == layer) {
                    c2 = cb + flt_wire(T, layer - 1, minx, maxx, miny, maxy);
                } else if (far) {
                    const int seq = (layer - 1) * 9 + (tl - 1);
                    const double c_e = F.ce[size_t(e) * 81 + seq];
                    if (!(c_e < kInf)) continue;
                    c2 = cb + c_e;
                    choice = seq;
                } else {
                    continue;
                }
                const unsigned long long v = flt_pack(static_cast<float>(c2), i * 100 + choice);
                if (v < cache[tl]) cache[tl] = v;
            }
        }
        for (int tl = 1; tl < kFltLayers; ++tl) atomicMin(ppk + tl, cache[tl]);
    }
}

// trace_flt_node (flt_block.cuh:144-331) for net-local node `i`: sets lo[i]
// and writes up to 4 segments (8 words) into `w`; returns the word count.
__device__ __forceinline__ int flt_trace_node(const Tables& T, const Flt& F, int nb, int eb, int i, int* w) {
    const int g = nb + i;
    const int c0 = F.coord[g];
    const int cx = c0 / T.Y % T.X, cy = c0 % T.Y, l = c0 / T.XY;
    const int pb = i ? F.pend[g - 1] : 0, pe = F.pend[g];
    int n = 0;
    int me;
    if (pb == pe) {
        int ml = 0;
        double mc = F.costs[size_t(g) * kFltLayers];
        for (int layer = 1; layer < kFltLayers; ++layer) {
            const double v = F.costs[size_t(g) * kFltLayers + layer];
            if (v < mc) { mc = v; ml = layer; }
        }
        me = ml;
    } else {
        int par_layer = -1, par_idx = -1, par_edge = -1;
        me = -1;
        for (int e = eb + pb; e < eb + pe; ++e) {
            const int pn = nb + F.eparent[e];
            const int pl = F.lo[pn];
            if (pl <= 0) continue;
            par_idx = pn; par_edge = e; par_layer = pl;
            const unsigned long long path = F.best[(size_t(F.child_off[pn]) + F.eslot[e] % 10) * kFltLayers + pl];
            const unsigned long long cidx = path / kFltLayers / 100, choice = (path / kFltLayers) % 100;
            if (cidx != static_cast<unsigned long long>(i)) { me = -1; continue; }
            me = choice == kFltStraight ? int(path % kFltLayers) : int(choice / 9 + 1);
            const int cpp = F.coord[pn], px = cpp / T.Y % T.X, py = cpp % T.Y;
            const bool vert = px == cx && cy != py, horz = py == cy && cx != px;
            if (vert || horz) {
                if (choice == kFltStraight) {
                    const int ll = me - 1;
                    if (vert) { w[n++] = cell_index(T, ll, px, min(py, cy)); w[n++] = cell_index(T, ll, px, max(py, cy)); }
                    else { w[n++] = cell_index(T, ll, min(px, cx), py); w[n++] = cell_index(T, ll, max(px, cx), py); }
                } else {
                    const int fl = int(choice / 9), tl = int(choice % 9);
                    const int cp = F.bc[size_t(e) * 81 + fl * 9 + tl];
                    if (vert) {
                        w[n++] = cell_index(T, fl, cx, min(cy, cp)); w[n++] = cell_index(T, fl, cx, max(cy, cp));
                        w[n++] = cell_index(T, min(fl, tl), cx, cp); w[n++] = cell_index(T, max(fl, tl), cx, cp);
                        w[n++] = cell_index(T, tl, cx, min(py, cp)); w[n++] = cell_index(T, tl, cx, max(py, cp));
                    } else {
                        w[n++] = cell_index(T, fl, min(cx, cp), cy); w[n++] = cell_index(T, fl, max(cx, cp), cy);
                        w[n++] = cell_index(T, min(fl, tl), cp, cy); w[n++] = cell_index(T, max(fl, tl), cp, cy);
                        w[n++] = cell_index(T, tl, min(px, cp), cy); w[n++] = cell_index(T, tl, max(px, cp), cy);
                    }
                }
            }
            break;
        }
        if (par_layer == -1) { F.lo[g] = -1; return 0; }
        const unsigned long long path =
            F.best[(size_t(F.child_off[par_idx]) + F.eslot[par_edge] % 10) * kFltLayers + par_layer];
        if (path / kFltLayers / 100 != static_cast<unsigned long long>(i)) { F.lo[g] = -1; return 0; }
    }
    F.lo[g] = me;
    int minl = l + 1, maxl = (l + 1) == kFltLayers ? 1 : minl;
    minl = min(minl, me);
    maxl = max(maxl, me);
    const int nc = F.children[g];
    for (int c = 0; c < nc; ++c) {
        const int lc = int(F.best[(size_t(F.child_off[g]) + c) * kFltLayers + me] % kFltLayers);
        minl = min(lc, minl);
        maxl = max(lc, maxl);
    }
    if (minl < 1) return -1;  // no finite layer at the root
    if (minl < maxl) { w[n++] = cell_index(T, minl - 1, cx, cy); w[n++] = cell_index(T, maxl - 1, cx, cy); }
    return n;
}

// Route net `id` with one warp: tables, solve, trace into the phase-two
// routes, then (if `commit`) its wire demand.  P2 is the phase-two view of the
// plan (routes = routes2).  All 32 lanes call with the same id.
__device__ __forceinline__ void flt_net(const Tables& T, const Flt& F, const Plan& P2, int id, int stamp, int lane,
                                        bool commit) {
    const int nb = F.node_off[id], N = F.node_off[id + 1] - nb;
    const int eb = F.edge_off[id];
    if (N <= 0) return;
    for (int k = lane; k < N * kFltLayers; k += 32) F.costs[size_t(nb) * kFltLayers + k] = kInf;
    const int cb = F.child_off[nb], cn = F.child_off[nb + N - 1] + F.children[nb + N - 1] - cb;
    for (int k = lane; k < cn * kFltLayers; k += 32) F.packed[size_t(cb) * kFltLayers + k] = kFltInit;
    __syncwarp();
    const int* lev = F.level + F.lvl_off[id];
    const int nl = F.lvl_off[id + 1] - F.lvl_off[id] - 1;
    const int* ord = F.order + nb;
    for (int d = nl - 1; d >= 0; --d) {
        for (int k = lev[d] + lane; k < lev[d + 1]; k += 32) flt_solve_node(T, F, nb, eb, ord[k]);
        __syncwarp();
    }
    int* r = F.routes2 + P2.route_off[id];
    const long long cap = P2.route_off[id + 1] - P2.route_off[id];
    long long count = 1;
    bool bad = false;
    for (int d = 0; d < nl; ++d) {
        for (int base = lev[d]; base < lev[d + 1]; base += 32) {
            int w[8];
            int n = 0;
            if (base + lane < lev[d + 1]) n = flt_trace_node(T, F, nb, eb, ord[base + lane], w);
            if (__any_sync(0xffffffffu, n < 0)) { bad = true; n = max(n, 0); }
            int off = n;
            for (int s = 1; s < 32; s <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, off, s);
                if (lane >= s) off += v;
            }
            const int total = __shfl_sync(0xffffffffu, off, 31);
            off -= n;
            if (count + total <= cap)
                for (int k = 0; k < n; ++k) r[count + off + k] = w[k];
            else bad = true;
            count += total;
            __syncwarp();
        }
    }
    if (lane == 0) {
        if (bad) { set_error(T, kELimit, id); r[0] = 1; }
        else r[0] = int(count);
    }
    __syncwarp();
    if (commit && !bad) commit_net_wires(T, P2, id, stamp, 1, lane);
}

// Route net `id` with the whole CTA: flt_net for nets whose DAG has a level
// wider than a warp, the CTA's threads over a level's nodes.  The words go
// out in the same order (level by level, ascending node index, each node's
// wires before its via stack): a block scan of the words per node replaces
// the warp scan.  All threads of the CTA call with the same id.
__device__ __forceinline__ void flt_net_block(const Tables& T, const Flt& F, const Plan& P2, int id, int stamp,
                                              bool commit) {
    __shared__ int wsum[32];
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
    const int nb = F.node_off[id], N = F.node_off[id + 1] - nb;
    const int eb = F.edge_off[id];
    if (N <= 0) return;
    for (int k = tid; k < N * kFltLayers; k += nth) F.costs[size_t(nb) * kFltLayers + k] = kInf;
    const int cb = F.child_off[nb], cn = F.child_off[nb + N - 1] + F.children[nb + N - 1] - cb;
    for (int k = tid; k < cn * kFltLayers; k += nth) F.packed[size_t(cb) * kFltLayers + k] = kFltInit;
    __syncthreads();
    const int* lev = F.level + F.lvl_off[id];
    const int nl = F.lvl_off[id + 1] - F.lvl_off[id] - 1;
    const int* ord = F.order + nb;
    for (int d = nl - 1; d >= 0; --d) {
        for (int k = lev[d] + tid; k < lev[d + 1]; k += nth) flt_solve_node(T, F, nb, eb, ord[k]);
        __syncthreads();
    }
    int* r = F.routes2 + P2.route_off[id];
    const long long cap = P2.route_off[id + 1] - P2.route_off[id];
    long long count = 1;
    bool bad = false;
    for (int d = 0; d < nl; ++d) {
        for (int base = lev[d]; base < lev[d + 1]; base += nth) {
            int w[8];
            int n = 0;
            if (base + tid < lev[d + 1]) n = flt_trace_node(T, F, nb, eb, ord[base + tid], w);
            const bool neg = n < 0;
            n = max(n, 0);
            int off = n;  // inclusive scan inside the warp
            for (int s = 1; s < 32; s <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, off, s);
                if (lane >= s) off += v;
            }
            if (lane == 31) wsum[warp] = off;
            if (__syncthreads_or(neg)) bad = true;
            if (warp == 0) {  // inclusive scan of the warp totals
                int v = lane < nw ? wsum[lane] : 0;
                for (int s = 1; s < 32; s <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, v, s);
                    if (lane >= s) v += u;
                }
                if (lane < nw) wsum[lane] = v;
            }
            __syncthreads();
            const int total = wsum[nw - 1];
            off += (warp ? wsum[warp - 1] : 0) - n;
            if (count + total <= cap)
                for (int k = 0; k < n; ++k) r[count + off + k] = w[k];
            else bad = true;
            count += total;
            __syncthreads();  // wsum is reused by the next round
        }
    }
    if (tid == 0) {
        if (bad) { set_error(T, kELimit, id); r[0] = 1; }
        else r[0] = int(count);
    }
    __syncthreads();
    if (commit && !bad) commit_net_wires(T, P2, id, stamp, 1, lane, warp, nw);
}

}  // namespace grb
