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

extern "C" {

int grb_stage_traffic(const grb_grid* g, int32_t n_batches, const int32_t* batch_off, const int32_t* ids,
                       const int32_t* node_off, const int32_t* nodes, const int32_t* parents,
                       const int64_t* route_off, const int32_t* routes,
                       const int32_t* point_off, const int32_t* hseg_off, const int32_t* hsegs,
                       const int32_t* vseg_off, const int32_t* vsegs, int32_t sparsity, double* out) {
    if (!g || !out) return GRB_EINVAL;
    const int X = g->X, Y = g->Y, XY = X * Y, L = g->L, DIR = g->DIR;
    auto along_y = [&](int l) { return ((l & 1) ^ DIR) != 0; };
    auto idx = [&](int l, int x, int y) { return (l * X + x) * Y + y; };
    const size_t cells = size_t(L) * XY;
    double refresh = 0, dp = 0, commit = 0, batching = 0;
    // Cost refresh: batch 0 recomputes everything; later batches what the
    // previous batch's commit touched.
    std::vector<uint8_t> wire_dirty(cells, 0), via_dirty(cells, 0);
    std::vector<uint8_t> track_dirty;
    std::vector<int> track_base(L + 1, 0);
    for (int l = 0; l < L; ++l) track_base[l + 1] = track_base[l] + (along_y(l) ? X : Y);
    track_dirty.assign(track_base[L], 0);
    std::vector<int> touched;
    auto touch_edge = [&](int c) {
        const int l = c / XY, x = c / Y % X, y = c % Y;
        const bool ay = along_y(l);
        const int pos = ay ? y : x, len = ay ? Y : X, stride = ay ? 1 : Y;
        if (!wire_dirty[c]) { wire_dirty[c] = 1; touched.push_back(c); }
        if (!via_dirty[c]) { via_dirty[c] = 1; touched.push_back(c); }
        if (pos + 1 < len && !via_dirty[c + stride]) { via_dirty[c + stride] = 1; touched.push_back(c + stride); }
        track_dirty[track_base[l] + (ay ? x : y)] = 1;
    };
    std::vector<int32_t> ts(cells, 0);
    for (int b = 0; b < n_batches; ++b) {
        if (b == 0) {
            refresh += 12.0 * cells + 20.0 * cells + 12.0 * cells;
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
        const int stamp = b + 1;
        for (int k = batch_off[b]; k < batch_off[b + 1]; ++k) {
            const int id = ids[k];
            // DP reads: distinct prefix and via-cost entries of this net.
            std::vector<int> pre, via;
            const int N = node_off[id + 1] - node_off[id];
            const int* nd = nodes + node_off[id];
            const int* par = parents + node_off[id];
            for (int i = 0; i < N; ++i) {
                const int r = nd[i] % XY, x = r / Y, y = r % Y;
                for (int l = 0; l < L; ++l) via.push_back(l * XY + r);
                if (!i) continue;
                const int pr = nd[par[i]] % XY, px = pr / Y, py = pr % Y;
                const int mnx = std::min(x, px), mxx = std::max(x, px), mny = std::min(y, py), mxy = std::max(y, py);
                for (int l = 0; l < L; ++l) {
                    const bool ay = along_y(l);
                    if (x == px || y == py) {
                        if (ay ? x == px : y == py) { pre.push_back(idx(l, mxx, mxy)); pre.push_back(idx(l, mnx, mny)); }
                    } else {
                        if (ay) {
                            pre.push_back(idx(l, x, mxy)); pre.push_back(idx(l, x, mny));
                            pre.push_back(idx(l, px, mxy)); pre.push_back(idx(l, px, mny));
                        } else {
                            pre.push_back(idx(l, mxx, y)); pre.push_back(idx(l, mnx, y));
                            pre.push_back(idx(l, mxx, py)); pre.push_back(idx(l, mnx, py));
                        }
                        via.push_back(idx(l, x, py)); via.push_back(idx(l, px, y));
                    }
                }
            }
            std::sort(pre.begin(), pre.end()); pre.erase(std::unique(pre.begin(), pre.end()), pre.end());
            std::sort(via.begin(), via.end()); via.erase(std::unique(via.begin(), via.end()), via.end());
            const int32_t* rr = routes + route_off[id];
            dp += 8.0 * pre.size() + 4.0 * via.size() + 8.0 * N + 4.0 * rr[0];
            // Wire commit.
            for (int i = 1; i < rr[0]; i += 2) {
                const int a = rr[i], bb = rr[i + 1], layer = a / XY;
                if (layer != bb / XY) continue;
                const int x0 = a / Y % X, y0 = a % Y, x1 = bb / Y % X, y1 = bb % Y;
                const bool ay = x0 == x1;
                const int lo = ay ? std::min(y0, y1) : std::min(x0, x1), hi = ay ? std::max(y0, y1) : std::max(x0, x1);
                ts[a] = ts[bb] = stamp;
                for (int pos = lo; pos < hi; ++pos) {
                    const int c = layer * XY + (ay ? x0 * Y + pos : pos * Y + y0);
                    ts[c] = stamp;
                    commit += 12.0;
                    touch_edge(c);
                }
            }
        }
        for (int k = batch_off[b]; k < batch_off[b + 1]; ++k) {
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
    out[0] = refresh; out[1] = dp; out[2] = commit; out[3] = batching;
    return GRB_OK;
}

}  // extern "C"
