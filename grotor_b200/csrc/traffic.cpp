// traffic.cpp -- algorithmic (compulsory) byte counts of a routing stage.
//
// Host-side measurement helper: the roofline of each kernel divides these
// bytes by the kernel's measured time.  The counts follow the model stated in
// include/grb_prof.h; they depend only on the plan, the topology and the
// stage's routes, never on how a kernel happens to move data.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/grb_prof.h"

namespace {

// The refresh / commit part of the byte model, shared by the stages: dirty
// cells and tracks since the last refresh, and the commit bytes of route
// words (wires, then vias that no wire of the same stamp covers).
struct StageModel {
    const grb_grid* g;
    int X, Y, XY, L, DIR;
    std::vector<uint8_t> wire_dirty, via_dirty, track_dirty;
    std::vector<int> track_base, touched;
    std::vector<int32_t> ts;
    double refresh = 0, commit = 0;
    bool first = true;
    explicit StageModel(const grb_grid* gg) : g(gg), X(gg->X), Y(gg->Y), XY(gg->X * gg->Y), L(gg->L), DIR(gg->DIR) {
        const size_t cells = size_t(L) * XY;
        wire_dirty.assign(cells, 0);
        via_dirty.assign(cells, 0);
        ts.assign(cells, 0);
        track_base.assign(L + 1, 0);
        for (int l = 0; l < L; ++l) track_base[l + 1] = track_base[l] + (along_y(l) ? X : Y);
        track_dirty.assign(track_base[L], 0);
    }
    bool along_y(int l) const { return ((l & 1) ^ DIR) != 0; }
    void touch_edge(int c) {
        const int l = c / XY, x = c / Y % X, y = c % Y;
        const bool ay = along_y(l);
        const int pos = ay ? y : x, len = ay ? Y : X, stride = ay ? 1 : Y;
        if (!wire_dirty[c]) { wire_dirty[c] = 1; touched.push_back(c); }
        if (!via_dirty[c]) { via_dirty[c] = 1; touched.push_back(c); }
        if (pos + 1 < len && !via_dirty[c + stride]) { via_dirty[c + stride] = 1; touched.push_back(c + stride); }
        track_dirty[track_base[l] + (ay ? x : y)] = 1;
    }
    // One refresh_cost: the first counts every cell and track.
    void refresh_now() {
        const double cells = double(L) * XY;
        if (first) {
            refresh += 12.0 * cells + 20.0 * cells + 12.0 * cells;
            first = false;
        } else {
            double wd = 0, vd = 0, td = 0;
            for (int c : touched) { wd += wire_dirty[c]; vd += via_dirty[c]; }
            for (int l = 0; l < L; ++l)
                for (int t = track_base[l]; t < track_base[l + 1]; ++t)
                    if (track_dirty[t]) { td += along_y(l) ? Y : X; track_dirty[t] = 0; }
            refresh += 12.0 * wd + 20.0 * vd + 12.0 * td;
        }
        for (int c : touched) { wire_dirty[c] = 0; via_dirty[c] = 0; }
        touched.clear();
    }
    // Wire then via commit of the route words of nets ids[lo, hi) under `stamp`.
    void commit_nets(const int32_t* ids, int lo, int hi, const int64_t* route_off, const int32_t* routes, int stamp) {
        for (int k = lo; k < hi; ++k) {
            const int32_t* rr = routes + route_off[ids[k]];
            for (int i = 1; i < rr[0]; i += 2) {
                const int a = rr[i], bb = rr[i + 1], layer = a / XY;
                if (layer != bb / XY) continue;
                const int x0 = a / Y % X, y0 = a % Y, x1 = bb / Y % X, y1 = bb % Y;
                const bool ay = x0 == x1;
                const int p0 = ay ? std::min(y0, y1) : std::min(x0, x1), p1 = ay ? std::max(y0, y1) : std::max(x0, x1);
                ts[a] = ts[bb] = stamp;
                for (int pos = p0; pos < p1; ++pos) {
                    const int c = layer * XY + (ay ? x0 * Y + pos : pos * Y + y0);
                    ts[c] = stamp;
                    commit += 12.0;
                    touch_edge(c);
                }
            }
        }
        for (int k = lo; k < hi; ++k) {
            const int32_t* rr = routes + route_off[ids[k]];
            for (int i = 1; i < rr[0]; i += 2) {
                const int a = rr[i], bb = rr[i + 1];
                const int low = std::min(a / XY, bb / XY), high = std::max(a / XY, bb / XY);
                if (low == high) continue;
                const int x = a / Y % X, y = a % Y;
                for (int layer = low; layer < high; ++layer) {
                    const int c = layer * XY + x * Y + y;
                    if (ts[c] >= stamp) continue;
                    const bool ay = along_y(layer);
                    const int pos = ay ? y : x, len = ay ? Y : X, stride = ay ? 1 : Y;
                    if (!pos) { commit += 8; touch_edge(c); }
                    else if (pos == len - 1) { commit += 8; touch_edge(c - stride); }
                    else { commit += 16; touch_edge(c - stride); touch_edge(c); }
                }
            }
        }
    }
    int idx(int l, int x, int y) const { return (l * X + x) * Y + y; }
};

double dedup(std::vector<int>& v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    return double(v.size());
}

}  // namespace

extern "C" {

int grb_stage_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                       const int32_t* node_off, const int32_t* nodes, const int32_t* parents,
                       const int64_t* route_off, const int32_t* routes,
                       const int32_t* point_off, const int32_t* hseg_off, const int32_t* hsegs,
                       const int32_t* vseg_off, const int32_t* vsegs, int32_t sparsity, double* out) {
    if (!g || !out) return GRB_EINVAL;
    StageModel M(g);
    const int L = M.L, XY = M.XY, Y = M.Y;
    double dp = 0, batching = 0;
    std::vector<int> pre, via;
    for (int b = 0; b < n_batches; ++b) {
        M.refresh_now();
        for (int k = batch_off[b]; k < batch_off[b + 1]; ++k) {
            const int id = ids[k];
            // DP reads: distinct prefix and via-cost entries of this net.
            pre.clear();
            via.clear();
            const int N = node_off[id + 1] - node_off[id];
            const int* nd = nodes + node_off[id];
            const int* par = parents + node_off[id];
            for (int i = 0; i < N; ++i) {
                const int r = nd[i] % XY, x = r / Y, y = r % Y;
                for (int l = 0; l < L; ++l) via.push_back(l * XY + r);
                if (!i) continue;
                const int pr = nd[par[i]] % XY, px = pr / Y, py = pr % Y;
                for (int l = 0; l < L; ++l) {
                    if (x == px || y == py) {
                        if (M.along_y(l) ? x == px : y == py) { pre.push_back(M.idx(l, x, y)); pre.push_back(M.idx(l, px, py)); }
                    } else {
                        // both bends: the four corners of the edge's box
                        pre.push_back(M.idx(l, x, y)); pre.push_back(M.idx(l, x, py));
                        pre.push_back(M.idx(l, px, y)); pre.push_back(M.idx(l, px, py));
                        via.push_back(M.idx(l, x, py)); via.push_back(M.idx(l, px, y));
                    }
                }
            }
            const int32_t* rr = routes + route_off[id];
            dp += 8.0 * dedup(pre) + 4.0 * dedup(via) + 8.0 * N + 4.0 * rr[0];
        }
        M.commit_nets(ids, batch_off[b], batch_off[b + 1], route_off, routes, b + 1);
    }
    // Batching: query points, marked cells, per-net mask and batch id.
    const int n = n_batches ? batch_off[n_batches] : 0;
    for (int k = 0; k < n; ++k) {
        const int id = ids[k];
        double marks = 4.0 * (point_off[id + 1] - point_off[id]);
        for (int s = hseg_off[id]; s < hseg_off[id + 1]; ++s)
            if (hsegs[2 * s + 1] >= hsegs[2 * s]) marks += (hsegs[2 * s + 1] - hsegs[2 * s]) / (sparsity * Y) + 1;
        for (int s = vseg_off[id]; s < vseg_off[id + 1]; ++s)
            if (vsegs[2 * s + 1] >= vsegs[2 * s]) marks += (vsegs[2 * s + 1] - vsegs[2 * s]) / sparsity + 1;
        batching += 4.0 * (point_off[id + 1] - point_off[id]) + 4.0 * marks + 132.0;
    }
    out[0] = M.refresh; out[1] = dp; out[2] = M.commit; out[3] = batching;
    return GRB_OK;
}


int grb_zshape_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                       const int32_t* node_off, const int32_t* coord, const int32_t* child,
                       const int64_t* route_off, const int32_t* routes, double* out) {
    if (!g || !out) return GRB_EINVAL;
    StageModel M(g);
    const int L = M.L, XY = M.XY, Y = M.Y;
    double dp = 0;
    std::vector<int> pre, via;
    for (int b = 0; b < n_batches; ++b) {
        M.refresh_now();
        for (int k = batch_off[b]; k < batch_off[b + 1]; ++k) {
            const int id = ids[k], nb = node_off[id], N = node_off[id + 1] - nb;
            pre.clear();
            via.clear();
            for (int i = 0; i < N; ++i) {
                const int r = coord[nb + i] % XY, tx = r / Y, ty = r % Y;
                for (int l = 0; l < L; ++l) via.push_back(M.idx(l, tx, ty));
                for (int j = 0; j < 3; ++j) {
                    const int ch = child[3 * (size_t(nb) + i) + j];
                    if (ch < 0) continue;
                    const int rc = coord[nb + ch] % XY, fx = rc / Y, fy = rc % Y;
                    const int mnx = std::min(fx, tx), mxx = std::max(fx, tx), mny = std::min(fy, ty), mxy = std::max(fy, ty);
                    if (fx != tx && fy != ty) {
                        // every layer: the box's two rows and two columns (wire
                        // prefixes and the via sweeps on them)
                        for (int l = 0; l < L; ++l) {
                            for (int x = mnx; x <= mxx; ++x) {
                                pre.push_back(M.idx(l, x, fy)); pre.push_back(M.idx(l, x, ty));
                                via.push_back(M.idx(l, x, fy)); via.push_back(M.idx(l, x, ty));
                            }
                            for (int y = mny; y <= mxy; ++y) {
                                pre.push_back(M.idx(l, fx, y)); pre.push_back(M.idx(l, tx, y));
                                via.push_back(M.idx(l, fx, y)); via.push_back(M.idx(l, tx, y));
                            }
                        }
                    } else {
                        for (int l = 0; l < L; ++l)
                            if (M.along_y(l) == (fx == tx)) { pre.push_back(M.idx(l, fx, fy)); pre.push_back(M.idx(l, tx, ty)); }
                    }
                }
            }
            const int32_t* rr = routes + route_off[id];
            dp += 8.0 * dedup(pre) + 4.0 * dedup(via) + 16.0 * N + 4.0 * rr[0];
        }
        M.commit_nets(ids, batch_off[b], batch_off[b + 1], route_off, routes, b + 1);
    }
    out[0] = M.refresh; out[1] = dp; out[2] = M.commit;
    return GRB_OK;
}

int grb_flt_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                    const grb_flt_dags* d, const int64_t* route_off, const int32_t* routes, const int32_t* routes2,
                    int32_t remove_phase_one, double* out) {
    if (!g || !d || !out) return GRB_EINVAL;
    StageModel M(g);
    const int L = M.L, XY = M.XY, Y = M.Y, X = M.X;
    double dp = 0;
    std::vector<int> pre, via;
    int stamp = 0;
    for (int b = 0; b < n_batches; ++b) {
        if (remove_phase_one) M.commit_nets(ids, batch_off[b], batch_off[b + 1], route_off, routes, ++stamp);
        ++stamp;
        M.refresh_now();
        for (int k = batch_off[b]; k < batch_off[b + 1]; ++k) {
            const int id = ids[k], nb = d->node_off[id], N = d->node_off[id + 1] - nb;
            const int eb = d->edge_off[id], E = d->edge_off[id + 1] - eb;
            pre.clear();
            via.clear();
            for (int i = 0; i < N; ++i) {
                const int r = d->coord[nb + i] % XY, x = r / Y, y = r % Y;
                for (int l = 0; l < L; ++l) via.push_back(M.idx(l, x, y));
            }
            for (int e = eb; e < eb + E; ++e) {
                const int to = nb + d->edge_parent[e], from = nb + d->edge_source_slot[e] / 10;
                const int ct = d->coord[to] % XY, cf = d->coord[from] % XY;
                const int tox = ct / Y, toy = ct % Y, fx = cf / Y, fy = cf % Y;
                // straight wires of the solve
                for (int l = 0; l < L; ++l)
                    if ((M.along_y(l) && fx == tox) || (!M.along_y(l) && fy == toy)) {
                        pre.push_back(M.idx(l, fx, fy)); pre.push_back(M.idx(l, tox, toy));
                    }
                // sampled layer changes (precompute_cost_edge)
                const int distance = std::abs(tox - fx) + std::abs(toy - fy);
                if (distance <= 4 || (fx != tox && fy != toy)) continue;
                const bool vertical = fx == tox;
                const int dd = distance / std::min(distance, 20);
                const int st = vertical ? std::min(fy, toy) : std::min(fx, tox), en = vertical ? std::max(fy, toy) : std::max(fx, tox);
                for (int sp = st + dd; sp < en; sp += dd) {
                    const int sx = vertical ? fx : sp, sy = vertical ? sp : fy;
                    for (int l = 0; l < L; ++l) {
                        if (M.along_y(l) != vertical) continue;
                        via.push_back(M.idx(l, sx, sy));
                        pre.push_back(M.idx(l, sx, sy));
                        pre.push_back(M.idx(l, vertical ? tox : sp, vertical ? sp : toy));
                    }
                }
            }
            (void)X;
            dp += 8.0 * dedup(pre) + 4.0 * dedup(via) + 20.0 * N + 8.0 * E + 4.0 * routes2[d->route2_off[id]];
        }
        M.commit_nets(ids, batch_off[b], batch_off[b + 1], d->route2_off, routes2, stamp);
    }
    out[0] = M.refresh; out[1] = dp; out[2] = M.commit;
    return GRB_OK;
}

int grb_dag_reads(const grb_grid* g, int32_t n, const int32_t* ids, const int32_t* node_off, const int32_t* nodes,
                  const int32_t* parents, double* out) {
    if (!g || !out) return GRB_EINVAL;
    StageModel M(g);
    const int L = M.L, XY = M.XY, Y = M.Y;
    double npre = 0, nvia = 0, nnodes = 0;
    std::vector<int> pre, via;
    for (int k = 0; k < n; ++k) {
        const int id = ids ? ids[k] : k;
        const int N = node_off[id + 1] - node_off[id];
        const int* nd = nodes + node_off[id];
        const int* par = parents + node_off[id];
        pre.clear();
        via.clear();
        for (int i = 0; i < N; ++i) {
            const int r = nd[i] % XY, x = r / Y, y = r % Y;
            for (int l = 0; l < L; ++l) via.push_back(l * XY + r);
            if (!i) continue;
            const int pr = nd[par[i]] % XY, px = pr / Y, py = pr % Y;
            for (int l = 0; l < L; ++l) {
                const bool ay = M.along_y(l);
                if (x == px || y == py) {
                    if (ay ? x == px : y == py) { pre.push_back(M.idx(l, x, y)); pre.push_back(M.idx(l, px, py)); }
                } else {
                    pre.push_back(M.idx(l, x, y)); pre.push_back(M.idx(l, x, py));
                    pre.push_back(M.idx(l, px, y)); pre.push_back(M.idx(l, px, py));
                    via.push_back(M.idx(l, x, py)); via.push_back(M.idx(l, px, y));
                }
            }
        }
        npre += dedup(pre);
        nvia += dedup(via);
        nnodes += N;
    }
    out[0] = npre; out[1] = nvia; out[2] = nnodes;
    return GRB_OK;
}

}  // extern "C"
