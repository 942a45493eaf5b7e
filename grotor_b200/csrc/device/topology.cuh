// topology.cuh -- every net's DP tree and batching geometry, built on the
// device from its Steiner tree.
//
// Semantics (the reference builds both on the host, 8 threads):
//   * geometry, net::construct_rsmt (preprocess.hpp:95-123): the points are
//     the nodes' 2-D cells in node order, then per tree edge (i, j) with j < i,
//     visited for i ascending and j in i's adjacency order: an edge with both
//     coordinates different adds the h-segments on rows min y and max y, the
//     v-segments on columns min x and max x and the two corner points
//     (xi, yj), (xj, yi); a horizontal edge adds its h-segment and its two
//     end points; a vertical one its v-segment and end points; an edge of
//     coincident nodes adds nothing;
//   * DP tree, the depth-first flattening of Lshape_route (lshape.cuh:85-98):
//     preorder from node 0, neighbours in adjacency order except the parent,
//     each node's 3-D position and its parent's preorder index (-1 at the
//     root).
//
// B200 form: one thread per net in two passes -- count (points, h- and
// v-segments per net, with the adjacency checked) and, after exclusive scans
// of the counts, fill.  The recursive DFS becomes an explicit stack in global
// scratch at three words per node of the net: a node's unvisited neighbours
// are pushed in reverse adjacency order, so they pop in adjacency order and
// each subtree is finished before the next sibling, which is the recursion's
// preorder.  A net whose adjacency is not a tree on its nodes (an index out of
// range, a node reached twice, a node never reached) is reported, not built.
#pragma once
#include "common.cuh"

namespace grb {

struct TopoBuild {
    int n, X, Y, L;
    long long nn, na;      // nodes, adjacency entries
    const int* node_off;   // [n+1]
    const int* pos;        // per node: layer*X*Y + x*Y + y (layer L: Steiner point)
    const int* adj_off;    // [nodes+1]
    const int* adj;        // net-local neighbour indices
    long long* cnt[3];     // points, h-segments, v-segments per net; scanned in place ([n] = total)
    int* nodes;
    int* parents;
    int* point_off; int* points;
    int* hseg_off;  int* hsegs;
    int* vseg_off;  int* vsegs;
    int* stack;            // [3 * nodes]
    int* seen;             // [nodes], zero before the fill
    int* status;           // [0] code (1 adjacency, 2 position, 3 not a tree), [1] net
};

__device__ __forceinline__ void topo_fail(const TopoBuild& B, int code, int net) {
    if (atomicCAS(B.status, 0, code) == 0) B.status[1] = net;
}

// The kind of tree edge (i, j): 0 none, 1 h and v (both coordinates differ),
// 2 horizontal (x differs), 3 vertical (y differs).
__device__ __forceinline__ int topo_edge_kind(int pi, int pj, int Y) {
    const int xi = pi / Y, yi = pi - xi * Y, xj = pj / Y, yj = pj - xj * Y;
    if (xi != xj && yi != yj) return 1;
    if (xi != xj) return 2;
    if (yi != yj) return 3;
    return 0;
}

// Pass 1: per net the number of points and segments; adjacency and positions
// checked.
__device__ __forceinline__ void topo_count(const TopoBuild& B, int id) {
    const int XY = B.X * B.Y;
    const int base = B.node_off[id], N = B.node_off[id + 1] - base;
    long long np = N, nh = 0, nv = 0;
    bool ok = base >= 0 && N >= 0 && base + static_cast<long long>(N) <= B.nn;
    if (!ok) topo_fail(B, 1, id);
    for (int i = 0; i < N && ok; ++i) {
        const int pi = B.pos[base + i];
        if (pi < 0 || pi / XY > B.L) { topo_fail(B, 2, id); ok = false; break; }
        const int a0 = B.adj_off[base + i], a1 = B.adj_off[base + i + 1];
        if (a0 < 0 || a1 < a0 || a1 > B.na) { topo_fail(B, 1, id); ok = false; break; }
        for (int k = a0; k < a1; ++k) {
            const int j = B.adj[k];
            if (j < 0 || j >= N) { topo_fail(B, 1, id); ok = false; break; }
            if (j >= i) continue;
            const int kind = topo_edge_kind(pi % XY, B.pos[base + j] % XY, B.Y);
            np += kind ? 2 : 0;
            nh += kind == 1 ? 2 : kind == 2 ? 1 : 0;
            nv += kind == 1 ? 2 : kind == 3 ? 1 : 0;
        }
    }
    B.cnt[0][id] = ok ? np : 0;
    B.cnt[1][id] = ok ? nh : 0;
    B.cnt[2][id] = ok ? nv : 0;
}

// Pass 2: geometry at the scanned offsets, then the depth-first flattening.
__device__ __forceinline__ void topo_fill(const TopoBuild& B, int id) {
    const int XY = B.X * B.Y, Y = B.Y;
    const int base = B.node_off[id], N = B.node_off[id + 1] - base;
    long long p = B.cnt[0][id], h = B.cnt[1][id], v = B.cnt[2][id];
    B.point_off[id] = static_cast<int>(p);
    B.hseg_off[id] = static_cast<int>(h);
    B.vseg_off[id] = static_cast<int>(v);
    if (id == B.n - 1) {
        B.point_off[B.n] = static_cast<int>(B.cnt[0][B.n]);
        B.hseg_off[B.n] = static_cast<int>(B.cnt[1][B.n]);
        B.vseg_off[B.n] = static_cast<int>(B.cnt[2][B.n]);
    }
    if (p == B.cnt[0][id + 1] && N > 0) return;  // failed the count (no points recorded)
    for (int i = 0; i < N; ++i) B.points[p++] = B.pos[base + i] % XY;
    for (int i = 0; i < N; ++i) {
        const int pi = B.pos[base + i] % XY, xi = pi / Y, yi = pi - xi * Y;
        for (int k = B.adj_off[base + i]; k < B.adj_off[base + i + 1]; ++k) {
            const int j = B.adj[k];
            if (j >= i) continue;
            const int pj = B.pos[base + j] % XY, xj = pj / Y, yj = pj - xj * Y;
            const int mnx = min(xi, xj), mxx = max(xi, xj), mny = min(yi, yj), mxy = max(yi, yj);
            switch (topo_edge_kind(pi, pj, Y)) {
                case 1:
                    B.hsegs[2 * h] = mnx * Y + mny; B.hsegs[2 * h + 1] = mxx * Y + mny; ++h;
                    B.hsegs[2 * h] = mnx * Y + mxy; B.hsegs[2 * h + 1] = mxx * Y + mxy; ++h;
                    B.vsegs[2 * v] = mnx * Y + mny; B.vsegs[2 * v + 1] = mnx * Y + mxy; ++v;
                    B.vsegs[2 * v] = mxx * Y + mny; B.vsegs[2 * v + 1] = mxx * Y + mxy; ++v;
                    B.points[p++] = xi * Y + yj;
                    B.points[p++] = xj * Y + yi;
                    break;
                case 2:
                    B.hsegs[2 * h] = mnx * Y + mny; B.hsegs[2 * h + 1] = mxx * Y + mny; ++h;
                    B.points[p++] = mnx * Y + mny;
                    B.points[p++] = mxx * Y + mny;
                    break;
                case 3:
                    B.vsegs[2 * v] = mnx * Y + mny; B.vsegs[2 * v + 1] = mnx * Y + mxy; ++v;
                    B.points[p++] = mnx * Y + mny;
                    B.points[p++] = mnx * Y + mxy;
                    break;
                default:
                    break;
            }
        }
    }
    if (N == 0) return;
    // Explicit-stack preorder: entries (node, parent node, parent's index).
    int* st = B.stack + 3 * static_cast<long long>(base);
    int top = 0, next = 0;
    st[0] = 0; st[1] = -1; st[2] = -1;
    top = 1;
    while (top > 0) {
        --top;
        const int x = st[3 * top], par = st[3 * top + 1], par_idx = st[3 * top + 2];
        if (next >= N || B.seen[base + x]) { topo_fail(B, 3, id); return; }
        B.seen[base + x] = 1;
        const int idx = next++;
        B.nodes[base + idx] = B.pos[base + x];
        B.parents[base + idx] = par_idx;
        const int a0 = B.adj_off[base + x], a1 = B.adj_off[base + x + 1];
        for (int k = a1 - 1; k >= a0; --k) {
            const int e = B.adj[k];
            if (e == par) continue;
            if (top >= N) { topo_fail(B, 3, id); return; }
            st[3 * top] = e; st[3 * top + 1] = x; st[3 * top + 2] = idx;
            ++top;
        }
    }
    if (next != N) topo_fail(B, 3, id);
}

}  // namespace grb
