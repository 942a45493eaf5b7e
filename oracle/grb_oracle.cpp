// grb_oracle.cpp -- CPU restatement of GRotor's routing hot path (test checker).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py, never by the product.  Each routine restates
// the reference's algorithm; citations are file:line in the GRotor project.
#include "grb_oracle.h"

#include <algorithm>
#include <functional>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kInf = 1e22;  // router_state.hpp:271

struct Grid {
    const orc_grid* g;
    int L, X, Y, DIR;
    explicit Grid(const orc_grid* p) : g(p), L(p->L), X(p->X), Y(p->Y), DIR(p->DIR) {}
    int idx(int l, int x, int y) const { return (l * X + x) * Y + y; }
    bool along_y(int l) const { return ((l & 1) ^ DIR) != 0; }
};

// The exponential of the cost model.  The reference evaluates CUDA's __expf;
// the host expf stands in for it (tolerance-level agreement), unless a table
// of the device's own values has been set (orc_set_exp_table): then every
// argument is looked up there and the cost tables come out bit-identical to
// the device's.  Arguments missing from a set table fall back to expf and are
// counted (orc_exp_table_misses), so a checker can prove the table was complete.
struct ExpTable {
    std::vector<float> x, y;  // x ascending
    std::atomic<long long> misses{0};
};
ExpTable g_exp;

float cost_exp(float a) {
    if (!g_exp.x.empty()) {
        const auto it = std::lower_bound(g_exp.x.begin(), g_exp.x.end(), a);
        if (it != g_exp.x.end() && *it == a) return g_exp.y[it - g_exp.x.begin()];
        g_exp.misses.fetch_add(1, std::memory_order_relaxed);
    }
    return expf(a);
}

// full_update.cuh:9-14 (of_cost_scaled).  The reference passes capacity and
// demand as float; the difference is a float subtraction, scaled in double, and
// the argument of the exponential is narrowed to float.  Returns false where
// no exponential is evaluated (zero capacity and no demand).
bool of_cost_arg(double scale, float capacity, float demand, float* arg) {
    if (capacity > 0.001) {
        const float diff = demand - capacity;
        const double a = 0.5 * static_cast<double>(diff);
        const double b = scale * 0.5 * static_cast<double>(diff);
        *arg = static_cast<float>(std::min(a, b));
        return true;
    }
    if (demand > 0) {
        const double a = 1.5 * static_cast<double>(demand);
        const double b = scale * 1.5 * static_cast<double>(demand);
        *arg = static_cast<float>(std::min(a, b));
        return true;
    }
    return false;
}

double of_cost_scaled(double scale, float capacity, float demand) {
    float a;
    return of_cost_arg(scale, capacity, demand, &a) ? static_cast<double>(cost_exp(a)) : 0.0;
}

// The demands incremental_of_cost passes to of_cost_scaled for a cell of
// demand h half-units: without and with each increment the cost model adds.
void cost_demands(int h, float out[3]) {
    const float dem = static_cast<float>(h) * 0.5f;
    out[0] = static_cast<float>(static_cast<double>(dem) + 0.0);
    out[1] = static_cast<float>(static_cast<double>(dem) + 1.0 + 0.0);
    out[2] = static_cast<float>(static_cast<double>(dem) + 0.5 + 0.0);
}

// full_update.cuh:23-32 (incremental_of_cost).
double incremental_of_cost(const Grid& G, const int32_t* demand_half, int l, int x, int y,
                           double incre, double base) {
    const int i = G.idx(l, x, y);
    const float cap = G.g->capacity[i];
    const float dem = static_cast<float>(demand_half[i]) * 0.5f;
    const float with = static_cast<float>(static_cast<double>(dem) + incre + base);
    const float without = static_cast<float>(static_cast<double>(dem) + base);
    const double delta = (of_cost_scaled(G.g->of_cost_scale, cap, with) -
                          of_cost_scaled(G.g->of_cost_scale, cap, without)) * G.g->short_costs[l];
    return std::min(1e12, delta);
}

// full_update.cuh:34-51 (update_single_wcost_ispd24).  The wire-length term is
// a multiply feeding an add, which the CUDA compiler contracts to one fma.
float wire_cost(const Grid& G, const int32_t* demand_half, int l, int x, int y) {
    float w = static_cast<float>(incremental_of_cost(G, demand_half, l, x, y, 1, 0));
    if (!G.along_y(l) && x < G.X - 1)
        w = static_cast<float>(std::fma(G.g->unit_wire, static_cast<double>(G.g->x_edge_len[x]), static_cast<double>(w)));
    if (G.along_y(l) && y < G.Y - 1)
        w = static_cast<float>(std::fma(G.g->unit_wire, static_cast<double>(G.g->y_edge_len[y]), static_cast<double>(w)));
    if (G.g->integer_wire) w = static_cast<float>(static_cast<int64_t>(std::fmin(std::fmax(w, 0.f), 1.e7f)));
    return w;
}

// full_update.cuh:58-83 (update_single_vcost_ispd24); cross points are 0 on
// one GPU (preprocess.hpp:1757).
float via_cost(const Grid& G, const int32_t* d, int l, int x, int y) {
    float v;
    if (G.along_y(l)) {
        if (y == 0) v = static_cast<float>(incremental_of_cost(G, d, l, x, y, 1, 0));
        else if (y == G.Y - 1) v = static_cast<float>(incremental_of_cost(G, d, l, x, y - 1, 1, 0));
        else v = static_cast<float>(incremental_of_cost(G, d, l, x, y, 0.5, 0) + incremental_of_cost(G, d, l, x, y - 1, 0.5, 0));
    } else {
        if (x == 0) v = static_cast<float>(incremental_of_cost(G, d, l, x, y, 1, 0));
        else if (x == G.X - 1) v = static_cast<float>(incremental_of_cost(G, d, l, x - 1, y, 1, 0));
        else v = static_cast<float>(incremental_of_cost(G, d, l, x, y, 0.5, 0) + incremental_of_cost(G, d, l, x - 1, y, 0.5, 0));
    }
    return static_cast<float>(static_cast<double>(v) + G.g->unit_via);
}

// One track of the prefix: shifted input s[0] = 0, s[i] = w[i-1]; output
// S(i) = sum_{j<=i} s[j] added exactly as the log-step scan of
// prefix_scan.cuh:84-95 adds it (equivalently the Fenwick rebuild of
// fenwick.cuh:146-166): for each set bit d of i, lowest first, add the total of
// the aligned 2^d block just below.  Block totals are pairwise sums, kept on a
// stack tot[d] = total of the most recently completed aligned 2^d block.
template <class T, class Load, class Store>
void sklansky_track(int n, Load load, Store store) {
    T tot[32];
    for (int i = 0; i < n; ++i) {
        T acc = i ? load(i - 1) : T(0);
        int d = 0;
        T fresh[32];
        fresh[0] = acc;
        while ((i >> d) & 1) {
            acc = acc + tot[d];
            ++d;
            fresh[d] = acc;
        }
        for (int j = 0; j <= d; ++j) tot[j] = fresh[j];
        for (int e = d + 1; (i >> e) != 0; ++e)
            if ((i >> e) & 1) acc = acc + tot[e];
        store(i, acc);
    }
}

}  // namespace

extern "C" {

int64_t orc_exp_args(const orc_grid* g, int32_t max_demand_half, float* out, int64_t cap) {
    std::vector<float> caps(g->capacity, g->capacity + size_t(g->L) * g->X * g->Y);
    std::sort(caps.begin(), caps.end());
    caps.erase(std::unique(caps.begin(), caps.end()), caps.end());
    std::vector<float> args;
    for (float c : caps)
        for (int h = 0; h <= max_demand_half; ++h) {
            float dem[3];
            cost_demands(h, dem);
            for (float d : dem) {
                float a;
                if (of_cost_arg(g->of_cost_scale, c, d, &a)) args.push_back(a);
            }
        }
    std::sort(args.begin(), args.end());
    args.erase(std::unique(args.begin(), args.end()), args.end());
    const int64_t n = int64_t(args.size());
    if (out) std::copy(args.begin(), args.begin() + std::min(n, cap), out);
    return n;
}

void orc_set_exp_table(int64_t n, const float* x, const float* y) {
    std::vector<std::pair<float, float>> v(size_t(std::max<int64_t>(n, 0)));
    for (int64_t i = 0; i < n; ++i) v[i] = {x[i], y[i]};
    std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    g_exp.x.resize(v.size());
    g_exp.y.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) { g_exp.x[i] = v[i].first; g_exp.y[i] = v[i].second; }
    g_exp.misses.store(0);
}

int64_t orc_exp_table_misses(void) { return g_exp.misses.load(); }

void orc_cost_full(const orc_grid* g, const int32_t* demand_half, float* wcost, float* vcost) {
    Grid G(g);
    const int cells = G.L * G.X * G.Y;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < cells; ++i) {
        const int l = i / (G.X * G.Y), x = i / G.Y % G.X, y = i % G.Y;
        if (wcost) wcost[i] = wire_cost(G, demand_half, l, x, y);
        if (vcost) vcost[i] = via_cost(G, demand_half, l, x, y);
    }
}

// prefix_scan.cuh:74-114 / fenwick.cuh:129-168: one track per (layer, row or
// column along the preferred direction).
void orc_presum(const orc_grid* g, const float* wcost, double* presum) {
    Grid G(g);
    for (int l = 0; l < G.L; ++l) {
        const bool ay = G.along_y(l);
        const int tracks = ay ? G.X : G.Y, len = ay ? G.Y : G.X, stride = ay ? 1 : G.Y;
#pragma omp parallel for schedule(static)
        for (int t = 0; t < tracks; ++t) {
            const int base = ay ? G.idx(l, t, 0) : G.idx(l, 0, t);
            sklansky_track<double>(len,
                [&](int k) { return static_cast<double>(wcost[base + k * stride]); },
                [&](int k, double v) { presum[base + k * stride] = v; });
        }
    }
}

// Literal log-step loop of prefix_scan.cuh:84-95.
void orc_presum_logstep(const orc_grid* g, const float* wcost, double* presum) {
    Grid G(g);
    std::vector<double> s;
    for (int l = 0; l < G.L; ++l) {
        const bool ay = G.along_y(l);
        const int tracks = ay ? G.X : G.Y, len = ay ? G.Y : G.X, stride = ay ? 1 : G.Y;
        s.assign(len, 0.0);
        for (int t = 0; t < tracks; ++t) {
            const int base = ay ? G.idx(l, t, 0) : G.idx(l, 0, t);
            s[0] = 0;
            for (int k = 0; k + 1 < len; ++k) s[k + 1] = wcost[base + k * stride];
            for (int d = 0; (1 << d) < len; ++d)
                for (int i = len - 1; i >= 0; --i)  // disjoint reads/writes per level
                    if ((i >> d) & 1) s[i] += s[((i >> d) << d) - 1];
            for (int k = 0; k < len; ++k) presum[base + k * stride] = s[k];
        }
    }
}

// lshape_thread.cuh:18-171 (Lshape_route_cuda), one net at a time; the warp
// kernel lshape_warp.cuh:105-247 is equal to it by construction (children of a
// parent are merged in descending node order in both).
int orc_lshape_batch(const orc_grid* g, const float* vcost, const double* presum,
                     int32_t n, const int32_t* ids, const int32_t* node_off,
                     const int32_t* nodes, const int32_t* parents,
                     const int64_t* route_off, int32_t* routes) {
    Grid G(g);
    const int L = G.L, X = G.X, Y = G.Y, DIR = G.DIR;
    int status = 0;
    auto wire = [&](int l, int xmin, int xmax, int ymin, int ymax) {  // prefix_scan.cuh:10-40
        return presum[G.idx(l, xmax, ymax)] - presum[G.idx(l, xmin, ymin)];
    };
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < n; ++k) {
        const int id = ids[k];
        const int N = node_off[id + 1] - node_off[id];
        const int* nd = nodes + node_off[id];
        const int* par = parents + node_off[id];
        std::vector<double> dist(size_t(N) * L * L);
        std::vector<int> from(size_t(N) * L * L, 0), range(N, 0);
        for (int i = 0; i < N; ++i) {
            const int l = nd[i] / X / Y, x = nd[i] / Y % X, y = nd[i] % Y;
            double* d = dist.data() + size_t(i) * L * L;
            for (int lo = 0; lo < L; ++lo) {
                d[lo * L + lo] = 0;
                for (int hi = lo + 1; hi < L; ++hi)
                    d[lo * L + hi] = d[lo * L + hi - 1] + static_cast<double>(vcost[G.idx(hi - 1, x, y)]);
                for (int hi = lo; hi < L; ++hi)
                    if (l < L && (lo > l || hi < l)) d[lo * L + hi] = kInf;
            }
        }
        for (int i = N - 1; i >= 1; --i) {
            const int x = nd[i] / Y % X, y = nd[i] % Y;
            const int p = par[i], px = nd[p] / Y % X, py = nd[p] % Y;
            const int minx = std::min(x, px), maxx = std::max(x, px), miny = std::min(y, py), maxy = std::max(y, py);
            const double* nd_dist = dist.data() + size_t(i) * L * L;
            double* par_dist = dist.data() + size_t(p) * L * L;
            int* prev = from.data() + size_t(i) * L * L;
            double cur[10], mcp[100];
            int cur_from[10] = {0};
            for (int l = 0; l < L; ++l) {
                cur[l] = mcp[l * L + l] = kInf;
                for (int lo = 0; lo <= l; ++lo)
                    for (int hi = l; hi < L; ++hi)
                        if (nd_dist[lo * L + hi] < cur[l]) { cur[l] = nd_dist[lo * L + hi]; cur_from[l] = lo * L + hi; }
            }
            if (x == px || y == py) {
                for (int l = 0; l < L; ++l) {
                    if (((l & 1) ^ DIR) == 0 && y != py) continue;
                    if (((l & 1) ^ DIR) == 1 && x != px) continue;
                    mcp[l * L + l] = cur[l] + wire(l, minx, maxx, miny, maxy);
                    prev[l * L + l] = cur_from[l] * L * L + l * L + l;
                }
            } else {
                for (int cl = 0; cl < L; ++cl) {
                    double cost = cur[cl];
                    if ((cl & 1) ^ DIR) cost += wire(cl, x, x, miny, maxy);
                    else cost += wire(cl, minx, maxx, y, y);
                    for (int pl = (cl & 1) ^ 1; pl < L; pl += 2) {
                        double cost2 = 0;
                        for (int l = std::min(cl, pl) + 1; l < std::max(cl, pl); ++l)
                            cost2 += ((cl & 1) ^ DIR) ? vcost[G.idx(l, x, py)] : vcost[G.idx(l, px, y)];
                        if ((pl & 1) ^ DIR) cost2 += wire(pl, px, px, miny, maxy);
                        else cost2 += wire(pl, minx, maxx, py, py);
                        if (cost + cost2 < mcp[pl * L + pl]) {
                            mcp[pl * L + pl] = cost + cost2;
                            prev[pl * L + pl] = cur_from[cl] * L * L + cl * L + pl;
                        }
                    }
                }
            }
            for (int lo = 0; lo < L; ++lo) {
                for (int hi = lo + 1; hi < L; ++hi) {
                    if (mcp[lo * L + hi - 1] <= mcp[hi * L + hi]) {
                        mcp[lo * L + hi] = mcp[lo * L + hi - 1];
                        prev[lo * L + hi] = prev[lo * L + hi - 1];
                    } else {
                        mcp[lo * L + hi] = mcp[hi * L + hi];
                        prev[lo * L + hi] = prev[hi * L + hi];
                    }
                }
                for (int hi = lo; hi < L; ++hi) par_dist[lo * L + hi] += mcp[lo * L + hi];
            }
        }
        // Root choice and traceback (lshape_thread.cuh:117-170).
        int32_t* out = routes + route_off[id];
        const int64_t cap = route_off[id + 1] - route_off[id];
        int64_t cnt = 1;
        bool overflow = false;
        auto emit = [&](int a, int b) {
            if (cnt + 2 > cap) { overflow = true; return; }
            out[cnt++] = a; out[cnt++] = b;
        };
        range[0] = 0;
        for (int lo = 0; lo < L; ++lo)
            for (int hi = lo; hi < L; ++hi)
                if (dist[lo * L + hi] < dist[range[0]]) range[0] = lo * L + hi;
        for (int i = 0; i < N; ++i) {
            const int* prev = from.data() + size_t(i) * L * L;
            if (i > 0) range[i] = prev[range[par[i]]] / L / L;
            const int minl = range[i] / L, maxl = range[i] % L, x = nd[i] / Y % X, y = nd[i] % Y;
            if (minl < maxl) emit(G.idx(minl, x, y), G.idx(maxl, x, y));
            if (i == 0) continue;
            const int px = nd[par[i]] / Y % X, py = nd[par[i]] % Y;
            const int minx = std::min(x, px), maxx = std::max(x, px), miny = std::min(y, py), maxy = std::max(y, py);
            const int cl = prev[range[par[i]]] / L % L, pl = prev[range[par[i]]] % L;
            if (px == x || py == y) {
                emit(G.idx(cl, minx, miny), G.idx(cl, maxx, maxy));
            } else if ((cl & 1) ^ DIR) {
                emit(G.idx(cl, x, y), G.idx(cl, x, py));
                emit(G.idx(cl, x, py), G.idx(pl, x, py));
                emit(G.idx(pl, x, py), G.idx(pl, px, py));
            } else {
                emit(G.idx(cl, x, y), G.idx(cl, px, y));
                emit(G.idx(cl, px, y), G.idx(pl, px, y));
                emit(G.idx(pl, px, y), G.idx(pl, px, py));
            }
        }
        if (cap > 0) out[0] = static_cast<int32_t>(cnt);
        if (overflow) {
#pragma omp critical
            if (!status) status = -1 - k;
        }
    }
    return status;
}

}  // extern "C"

namespace {
// demand.cuh:236-319 (commit_batch_wires then commit_batch_vias).  `touched`,
// when given, receives every edge cell whose demand changed.
void commit_impl(const orc_grid* g, int32_t n, const int32_t* ids,
                 const int64_t* route_off, const int32_t* routes,
                 int32_t stamp, int32_t K, int32_t* demand_half, int32_t* timestamp,
                 double* total_wirelength, int64_t* total_vias, std::vector<int>* touched) {
    Grid G(g);
    const int X = G.X, Y = G.Y, XY = X * Y;
    double length = 0;
    for (int k = 0; k < n; ++k) {
        const int32_t* r = routes + route_off[ids[k]];
        for (int i = 1; i < r[0]; i += 2) {
            const int a = r[i], b = r[i + 1], layer = a / XY;
            if (layer != b / XY) continue;
            const int x0 = a / Y % X, y0 = a % Y, x1 = b / Y % X, y1 = b % Y;
            const bool ay = x0 == x1;
            const int lo = ay ? std::min(y0, y1) : std::min(x0, x1);
            const int hi = ay ? std::max(y0, y1) : std::max(x0, x1);
            timestamp[a] = timestamp[b] = stamp;
            for (int pos = lo; pos < hi; ++pos) {
                const int index = layer * XY + (ay ? x0 * Y + pos : pos * Y + y0);
                demand_half[index] += 2 * K;
                timestamp[index] = stamp;
                if (touched) touched->push_back(index);
                length += ay ? g->y_edge_len[pos] : g->x_edge_len[pos];
            }
        }
    }
    int64_t vias = 0;
    for (int k = 0; k < n; ++k) {
        const int32_t* r = routes + route_off[ids[k]];
        for (int i = 1; i < r[0]; i += 2) {
            const int a = r[i], b = r[i + 1];
            const int low = std::min(a / XY, b / XY), high = std::max(a / XY, b / XY);
            if (low == high) continue;
            const int x = a / Y % X, y = a % Y;
            vias += high - low;
            for (int layer = low; layer < high; ++layer) {
                const int index = layer * XY + x * Y + y;
                if (timestamp[index] >= stamp) continue;
                const bool ay = G.along_y(layer);
                const int position = ay ? y : x, len = ay ? Y : X, stride = ay ? 1 : Y;
                if (!position) { demand_half[index] += 2 * K; if (touched) touched->push_back(index); }
                else if (position == len - 1) { demand_half[index - stride] += 2 * K; if (touched) touched->push_back(index - stride); }
                else {
                    demand_half[index - stride] += K; demand_half[index] += K;
                    if (touched) { touched->push_back(index - stride); touched->push_back(index); }
                }
            }
        }
    }
    if (total_wirelength) *total_wirelength += length * K;
    if (total_vias) *total_vias += vias * K;
}
}  // namespace

extern "C" {

void orc_commit_batch(const orc_grid* g, int32_t n, const int32_t* ids,
                      const int64_t* route_off, const int32_t* routes,
                      int32_t stamp, int32_t K, int32_t* demand_half, int32_t* timestamp,
                      double* total_wirelength, int64_t* total_vias) {
    commit_impl(g, n, ids, route_off, routes, stamp, K, demand_half, timestamp, total_wirelength, total_vias, nullptr);
}

// generate_batches_cpu.hpp:7-73 (generate_batches_rsmt).
int32_t orc_batches(int32_t X, int32_t Y, int32_t n, const int32_t* order,
                    const int32_t* point_off, const int32_t* points,
                    const int32_t* hseg_off, const int32_t* hsegs,
                    const int32_t* vseg_off, const int32_t* vsegs,
                    int32_t limit, int32_t sparsity, int32_t* batch_of) {
    std::vector<std::vector<uint8_t>> vis;
    std::vector<int32_t> size;
    for (int k = 0; k < n; ++k) {
        const int id = order[k];
        int bid = -1;
        for (int b = 0; b < static_cast<int>(vis.size()); ++b) {
            if (size[b] >= limit) continue;
            bool conflict = false;
            for (int q = point_off[id]; q < point_off[id + 1] && !conflict; ++q)
                conflict = vis[b][points[q]] != 0;
            if (!conflict) { bid = b; break; }
        }
        if (bid < 0) {
            bid = static_cast<int>(vis.size());
            vis.emplace_back(size_t(X) * Y, 0);
            size.push_back(0);
        }
        ++size[bid];
        batch_of[k] = bid;
        auto& v = vis[bid];
        for (int s = hseg_off[id]; s < hseg_off[id + 1]; ++s)
            for (int p = hsegs[2 * s]; p <= hsegs[2 * s + 1]; p += sparsity * Y) v[p] = 1;
        for (int s = vseg_off[id]; s < vseg_off[id + 1]; ++s)
            for (int p = vsegs[2 * s]; p <= vsegs[2 * s + 1]; p += sparsity) v[p] = 1;
        for (int q = point_off[id]; q < point_off[id + 1]; ++q) {
            const int px = points[q] / Y, py = points[q] % Y;
            for (int x = px - 1; x <= px + 1; ++x) {
                if (x < 0 || x >= X) continue;
                for (int y = py - 1; y < py + 1; ++y)  // y + 1 is not marked (reference :38)
                    if (y >= 0 && y < Y && (x == px || y == py)) v[size_t(x) * Y + y] = 1;
            }
        }
    }
    return static_cast<int32_t>(vis.size());
}

// congestion.cuh:8-58 and :114-136.
void orc_ripup_classify(const orc_grid* g, const int32_t* demand_half, int32_t threshold,
                        int32_t n_nets, const int64_t* route_off, const int32_t* routes,
                        uint8_t* is_of) {
    Grid G(g);
    const int cells = G.L * G.X * G.Y, X = G.X, Y = G.Y;
    std::vector<int> sum(cells, 0);
    for (int i = 0; i < cells; ++i) {
        const int l = i / (X * Y), x = i / Y % X, y = i % Y;
        if ((!G.along_y(l) && x + 1 < X) || (G.along_y(l) && y + 1 < Y))
            sum[i] = (g->capacity[i] + threshold <= static_cast<float>(demand_half[i]) * 0.5f) ? 1 : 0;
    }
    for (int l = 0; l < G.L; ++l) {  // prefix_scan.cuh:42-72 (integer scan, order-free)
        const bool ay = G.along_y(l);
        const int tracks = ay ? X : Y, len = ay ? Y : X, stride = ay ? 1 : Y;
        for (int t = 0; t < tracks; ++t) {
            const int base = ay ? G.idx(l, t, 0) : G.idx(l, 0, t);
            int acc = 0;
            for (int k = 0; k < len; ++k) {
                const int v = sum[base + k * stride];
                sum[base + k * stride] = acc;
                acc += v;
            }
        }
    }
    for (int id = 0; id < n_nets; ++id) {
        is_of[id] = 0;
        const int32_t* r = routes + route_off[id];
        int count = 0;
        for (int i = 1; i < r[0]; i += 2) {
            const int l = r[i] / X / Y, x0 = r[i] / Y % X, y0 = r[i] % Y;
            const int x1 = r[i + 1] / Y % X, y1 = r[i + 1] % Y;
            if (x0 != x1) count += sum[G.idx(l, std::max(x0, x1), y0)] - sum[G.idx(l, std::min(x0, x1), y0)];
            if (y0 != y1) count += sum[G.idx(l, x0, std::max(y0, y1))] - sum[G.idx(l, x0, std::min(y0, y1))];
            if (count > 10) { is_of[id] = 1; break; }
        }
    }
}

// congestion.cuh:60-112.
void orc_congestion_view(const orc_grid* g, const int32_t* demand_half,
                         uint8_t* congestion, float* xsum, float* ysum) {
    Grid G(g);
    const int X = G.X, Y = G.Y;
    std::vector<float> worst(size_t(X) * Y);
    for (int i = 0; i < X * Y; ++i) {
        double w = 0.0;
        for (int l = 0; l < G.L; ++l) {
            const int e = l * X * Y + i;
            w = std::max(w, static_cast<double>(static_cast<float>(demand_half[e]) * 0.5f - g->capacity[e]));
        }
        congestion[i] = w > 0.0;
        worst[i] = static_cast<float>(w);
    }
    for (int x = 0; x < X; ++x)  // extract_congestionView_ysum: per x, scan over y
        sklansky_track<float>(Y, [&](int k) { return worst[size_t(x) * Y + k]; },
                              [&](int k, float v) { ysum[size_t(x) * Y + k] = v; });
    for (int y = 0; y < Y; ++y)  // extract_congestionView_xsum: per y, scan over x
        sklansky_track<float>(X, [&](int k) { return worst[size_t(k) * Y + y]; },
                              [&](int k, float v) { xsum[size_t(k) * Y + y] = v; });
}

int orc_lshape_stage(const orc_grid* g, int32_t n_batches, const int32_t* batch_off,
                     const int32_t* ids, const int32_t* node_off, const int32_t* nodes,
                     const int32_t* parents, const int64_t* route_off, int32_t* routes,
                     int32_t* demand_half, int32_t* timestamp, int32_t* stamp,
                     double* total_wirelength, int64_t* total_vias, int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Grid G(g);
    const size_t cells = size_t(g->L) * g->X * g->Y;
    std::vector<float> wcost(cells), vcost(cells);
    std::vector<double> presum(cells);
    std::vector<int> touched;
    std::vector<uint8_t> wire_dirty(cells, 0), via_dirty(cells, 0);
    int status = 0;
    for (int b = 0; b < n_batches; ++b) {
        const int32_t s = ++*stamp;  // lshape.cuh:161
        // refresh_cost (incremental_update.cuh:98-132): the first refresh is
        // full; later ones recompute the cells the previous commit changed and
        // rescan their tracks (values identical to a full recompute).
        if (b == 0) {
            orc_cost_full(g, demand_half, wcost.data(), vcost.data());
            orc_presum(g, wcost.data(), presum.data());
        } else {
            std::vector<int> wlist, vlist;
            std::vector<int> tracks;
            for (int c : touched) {
                const int l = c / (G.X * G.Y), x = c / G.Y % G.X, y = c % G.Y;
                const bool ay = G.along_y(l);
                const int pos = ay ? y : x, len = ay ? G.Y : G.X, stride = ay ? 1 : G.Y;
                if (!wire_dirty[c]) { wire_dirty[c] = 1; wlist.push_back(c); }
                if (!via_dirty[c]) { via_dirty[c] = 1; vlist.push_back(c); }
                if (pos + 1 < len && !via_dirty[c + stride]) { via_dirty[c + stride] = 1; vlist.push_back(c + stride); }
            }
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < wlist.size(); ++k) {
                const int c = wlist[k];
                wcost[c] = wire_cost(G, demand_half, c / (G.X * G.Y), c / G.Y % G.X, c % G.Y);
            }
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < vlist.size(); ++k) {
                const int c = vlist[k];
                vcost[c] = via_cost(G, demand_half, c / (G.X * G.Y), c / G.Y % G.X, c % G.Y);
            }
            for (int c : wlist) {
                const int l = c / (G.X * G.Y), x = c / G.Y % G.X, y = c % G.Y;
                tracks.push_back(G.along_y(l) ? G.idx(l, x, 0) : G.idx(l, 0, y));
                wire_dirty[c] = 0;
            }
            for (int c : vlist) via_dirty[c] = 0;
            std::sort(tracks.begin(), tracks.end());
            tracks.erase(std::unique(tracks.begin(), tracks.end()), tracks.end());
#pragma omp parallel for schedule(dynamic, 4)
            for (size_t k = 0; k < tracks.size(); ++k) {
                const int base = tracks[k], l = base / (G.X * G.Y);
                const bool ay = G.along_y(l);
                const int len = ay ? G.Y : G.X, stride = ay ? 1 : G.Y;
                sklansky_track<double>(len,
                    [&](int q) { return static_cast<double>(wcost[base + q * stride]); },
                    [&](int q, double v) { presum[base + q * stride] = v; });
            }
        }
        touched.clear();
        const int n = batch_off[b + 1] - batch_off[b];
        const int rc = orc_lshape_batch(g, vcost.data(), presum.data(), n, ids + batch_off[b],
                                        node_off, nodes, parents, route_off, routes);
        if (rc && !status) status = rc;
        commit_impl(g, n, ids + batch_off[b], route_off, routes, s, 1, demand_half,
                    timestamp, total_wirelength, total_vias, &touched);
    }
    return status;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// FLT stage (flt.cuh:75-182, flt_cost.cuh:25-130, flt_block.cuh:6-355).
namespace {

constexpr int kFltLayers = 10;                         // MAX_LAYER, flt_cost.cuh:14
constexpr uint64_t kFltInit = 7208259049189261824ULL;  // init_cost_with_road, flt_cost.cuh:48
constexpr int kStraight = 82;                          // "no layer change" choice, flt_block.cuh:109

// flt_cost.cuh:25-46: a float cost in an order-preserving int32 in the high
// word, the candidate id in the low word.
int32_t flt_ordered(float f) {
    int32_t i;
    std::memcpy(&i, &f, 4);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
uint64_t flt_pack(float cost, int id) {
    return (uint64_t(uint32_t(flt_ordered(cost))) << 32) | uint32_t(id);
}
double flt_unpack_cost(uint64_t p) {
    int32_t i = int32_t(p >> 32);
    i = i >= 0 ? i : i ^ 0x7FFFFFFF;
    float f;
    std::memcpy(&f, &i, 4);
    return double(f);
}

// One net: layer-change tables, solve (deepest level first), trace (root
// first).  Nodes of one depth are visited in ascending node index, the order
// of the reference's stable depth sort (flt_workspace.cuh:216-217); the
// reference appends segments with atomics, so its order within a level may
// differ while the segment multiset is the same.
int flt_net(const Grid& G, const orc_flt* D, const float* vcost, const double* presum, int id,
            int32_t* r, int64_t cap) {
    const int nb = D->node_off[id], N = D->node_off[id + 1] - nb;
    const int eb = D->edge_off[id], E = D->edge_off[id + 1] - eb;
    if (N <= 0) return 0;
    const int X = G.X, Y = G.Y, XY = X * Y, L = G.L;
    const int* crd = D->coord + nb;
    const int* dep = D->depth + nb;
    const int* nch = D->children + nb;
    const int* pend = D->parent_end + nb;
    const int* epar = D->edge_parent + eb;
    const int* eslot = D->edge_slot + eb;
    auto wire = [&](int l, int xmin, int xmax, int ymin, int ymax) {  // prefix_scan.cuh:10-40
        return presum[G.idx(l, xmax, ymax)] - presum[G.idx(l, xmin, ymin)];
    };
    auto pbeg = [&](int i) { return i ? pend[i - 1] : 0; };
    std::vector<int> coff(N + 1, 0);
    int maxd = 0;
    for (int i = 0; i < N; ++i) { coff[i + 1] = coff[i] + nch[i]; maxd = std::max(maxd, dep[i]); }
    std::vector<int> lvl_off(maxd + 2, 0), order(N);
    for (int i = 0; i < N; ++i) ++lvl_off[dep[i] + 1];
    for (int d = 0; d <= maxd; ++d) lvl_off[d + 1] += lvl_off[d];
    {
        std::vector<int> fill(lvl_off.begin(), lvl_off.end() - 1);
        for (int i = 0; i < N; ++i) order[fill[dep[i]]++] = i;
    }
    // precompute_cost_edge (flt_cost.cuh:50-130): per edge and from-layer, the
    // best of <= 19 sampled change positions per same-parity to-layer.
    std::vector<double> ce(size_t(E) * 81, kInf);
    std::vector<int> bc(size_t(E) * 81, -1);
    for (int e = 0; e < E; ++e) {
        const int from = eslot[e] / 10, to = epar[e];
        const int tox = crd[to] / Y % X, toy = crd[to] % Y, fromx = crd[from] / Y % X, fromy = crd[from] % Y;
        for (int fl = 0; fl < 9; ++fl) {
            const bool ay = ((fl & 1) ^ G.DIR) != 0;
            if ((!ay && fromy != toy) || (ay && fromx != tox)) continue;  // rows stay INF
            const int distance = std::abs(tox - fromx) + std::abs(toy - fromy);
            if (!distance) continue;
            const int dd = distance / std::min(distance, 20);
            const bool vertical = fromx == tox;
            const int start = vertical ? std::min(fromy, toy) : std::min(fromx, tox);
            const int end = vertical ? std::max(fromy, toy) : std::max(fromx, tox);
            for (int tl = 0; tl < 9; ++tl) {
                if ((tl % 2) != (fl % 2)) continue;
                double best = kInf;
                int pos = -1;
                for (int sp = start + dd; sp < end; sp += dd) {
                    const int sx = vertical ? fromx : sp, sy = vertical ? sp : fromy;
                    double via = 0;
                    for (int ll = std::min(fl, tl); ll < std::max(fl, tl); ++ll) via += vcost[G.idx(ll, sx, sy)];
                    double c = via;
                    if (vertical)
                        c += (wire(fl, fromx, fromx, std::min(fromy, sy), std::max(fromy, sy)) +
                              wire(tl, tox, tox, std::min(toy, sy), std::max(toy, sy)));
                    else
                        c += (wire(fl, std::min(fromx, sx), std::max(fromx, sx), fromy, fromy) +
                              wire(tl, std::min(tox, sx), std::max(tox, sx), toy, toy));
                    if (c < best) { best = c; pos = sp; }
                }
                ce[size_t(e) * 81 + fl * 9 + tl] = best;
                bc[size_t(e) * 81 + fl * 9 + tl] = pos;
            }
        }
    }
    // solve_flt_node (flt_block.cuh:6-142).
    std::vector<double> costs(size_t(N) * kFltLayers, kInf);
    std::vector<uint64_t> packed(size_t(coff[N]) * kFltLayers, kFltInit), best(size_t(coff[N]) * kFltLayers, 0);
    for (int d = maxd; d >= 0; --d) {
        for (int k = lvl_off[d]; k < lvl_off[d + 1]; ++k) {
            const int node = order[k];
            const int flow = 1 + crd[node] / XY, x = crd[node] / Y % X, y = crd[node] % Y;
            const int fhigh = flow == kFltLayers ? 0 : flow;
            const int nc = nch[node];
            uint64_t* cbp = best.data() + size_t(coff[node]) * kFltLayers;
            const uint64_t* cpk = packed.data() + size_t(coff[node]) * kFltLayers;
            double* cst = costs.data() + size_t(node) * kFltLayers;
            double mcc[6];
            uint64_t bp[6] = {0, 0, 0, 0, 0, 0};
            for (int low = 1; low <= flow; ++low) {
                for (int c = 0; c < nc; ++c) mcc[c] = kInf;
                double via = 0;
                for (int li = low; li < L + 1; ++li) {
                    if (li > low) via += vcost[G.idx(li - 2, x, y)];
                    for (int c = 0; c < nc; ++c) {
                        const uint64_t pv = cpk[c * kFltLayers + li];
                        const double cc = flt_unpack_cost(pv);
                        if (cc < mcc[c]) { mcc[c] = cc; bp[c] = uint64_t(uint32_t(pv)) * kFltLayers + li; }
                    }
                    if (li >= fhigh) {
                        double cost = via;
                        for (int c = 0; c < nc; ++c) cost += mcc[c];
                        if (cost < kInf && cost < cst[li]) {
                            cst[li] = cost;
                            for (int c = 0; c < nc; ++c) cbp[c * kFltLayers + li] = bp[c];
                        }
                    }
                }
                for (int li = L - 1; li >= low; --li) {
                    if (cst[li + 1] < cst[li]) {
                        cst[li] = cst[li + 1];
                        for (int c = 0; c < nc; ++c) cbp[c * kFltLayers + li] = cbp[c * kFltLayers + li + 1];
                    }
                }
            }
            const int P = pend[node] - pbeg(node);
            for (int pi = 0; pi < P; ++pi) {
                const int e = pbeg(node) + pi, par = epar[e], slot = eslot[e] % 10;
                uint64_t* ppk = packed.data() + size_t(coff[par]) * kFltLayers;
                const int px = crd[par] / Y % X, py = crd[par] % Y;
                const int minx = std::min(x, px), maxx = std::max(x, px), miny = std::min(y, py), maxy = std::max(y, py);
                uint64_t cache[kFltLayers];
                for (int t = 0; t < kFltLayers; ++t) cache[t] = kFltInit;
                for (int layer = 1; layer < kFltLayers; ++layer) {
                    const bool ay = ((layer & 1) ^ G.DIR) == 1;  // 1-based layer index
                    if (ay && y != py) continue;
                    if (!ay && x != px) continue;
                    const double cb = cst[layer];
                    for (int tl = 1 + (1 - layer % 2); tl < kFltLayers; tl += 2) {
                        double c2;
                        int choice = kStraight;
                        if (tl == layer) c2 = cb + wire(layer - 1, minx, maxx, miny, maxy);
                        else if (std::abs(x - px) + std::abs(y - py) > 4) {
                            const int seq = (layer - 1) * 9 + (tl - 1);
                            const double c_e = ce[size_t(e) * 81 + seq];
                            if (!(c_e < kInf)) continue;
                            c2 = cb + c_e;
                            choice = seq;
                        } else continue;
                        const uint64_t v = flt_pack(static_cast<float>(c2), node * 100 + choice);
                        if (v < cache[tl]) cache[tl] = v;
                    }
                }
                for (int tl = 1; tl < kFltLayers; ++tl)
                    ppk[slot * kFltLayers + tl] = std::min(ppk[slot * kFltLayers + tl], cache[tl]);
            }
        }
    }
    // trace_flt_node (flt_block.cuh:144-331).
    std::vector<int> lo(N, -1);
    int status = 0;
    r[0] = 1;
    auto emit = [&](int a, int b) {
        if (r[0] + 2 > cap) { status = 3; return; }
        r[r[0]] = a;
        r[r[0] + 1] = b;
        r[0] += 2;
    };
    for (int d = 0; d <= maxd; ++d) {
        for (int k = lvl_off[d]; k < lvl_off[d + 1]; ++k) {
            const int node = order[k];
            const int cx = crd[node] / Y % X, cy = crd[node] % Y, l = crd[node] / XY;
            const int P = pend[node] - pbeg(node);
            if (P == 0) {
                int ml = 0;
                double mc = costs[size_t(node) * kFltLayers];
                for (int layer = 1; layer < kFltLayers; ++layer)
                    if (costs[size_t(node) * kFltLayers + layer] < mc) { mc = costs[size_t(node) * kFltLayers + layer]; ml = layer; }
                lo[node] = ml;
            } else {
                int par_layer = -1, par_idx = -1, par_seq = -1;
                for (int pi = 0; pi < P; ++pi) {
                    const int e = pbeg(node) + pi, pn = epar[e];
                    if (lo[pn] <= 0) continue;
                    par_idx = pn; par_seq = pi; par_layer = lo[pn];
                    const uint64_t path = best[size_t(coff[pn]) * kFltLayers + (eslot[e] % 10) * kFltLayers + par_layer];
                    const uint64_t cidx = path / kFltLayers / 100, choice = (path / kFltLayers) % 100;
                    if (cidx != uint64_t(node)) { lo[node] = -1; continue; }
                    lo[node] = choice == kStraight ? int(path % kFltLayers) : int(choice / 9 + 1);
                    const int px = crd[pn] / Y % X, py = crd[pn] % Y;
                    const bool vert = px == cx && cy != py, horz = py == cy && cx != px;
                    if (vert || horz) {
                        if (choice == kStraight) {
                            const int ll = lo[node] - 1;
                            if (vert) emit(G.idx(ll, px, std::min(py, cy)), G.idx(ll, px, std::max(py, cy)));
                            else emit(G.idx(ll, std::min(px, cx), py), G.idx(ll, std::max(px, cx), py));
                        } else {
                            const int fl = int(choice / 9), tl = int(choice % 9);
                            const int cp = bc[size_t(e) * 81 + fl * 9 + tl];
                            if (vert) {
                                emit(G.idx(fl, cx, std::min(cy, cp)), G.idx(fl, cx, std::max(cy, cp)));
                                emit(G.idx(std::min(fl, tl), cx, cp), G.idx(std::max(fl, tl), cx, cp));
                                emit(G.idx(tl, cx, std::min(py, cp)), G.idx(tl, cx, std::max(py, cp)));
                            } else {
                                emit(G.idx(fl, std::min(cx, cp), cy), G.idx(fl, std::max(cx, cp), cy));
                                emit(G.idx(std::min(fl, tl), cp, cy), G.idx(std::max(fl, tl), cp, cy));
                                emit(G.idx(tl, std::min(px, cp), cy), G.idx(tl, std::max(px, cp), cy));
                            }
                        }
                    }
                    break;
                }
                if (par_layer == -1) { lo[node] = -1; continue; }
                const int e = pbeg(node) + par_seq;
                const uint64_t path = best[size_t(coff[par_idx]) * kFltLayers + (eslot[e] % 10) * kFltLayers + par_layer];
                if (path / kFltLayers / 100 != uint64_t(node)) { lo[node] = -1; continue; }
            }
            int minl = l + 1, maxl = (l + 1) == kFltLayers ? 1 : minl;
            minl = std::min(minl, lo[node]);
            maxl = std::max(maxl, lo[node]);
            for (int c = 0; c < nch[node]; ++c) {
                const int lc = int(best[size_t(coff[node]) * kFltLayers + c * kFltLayers + lo[node]] % kFltLayers);
                minl = std::min(lc, minl);
                maxl = std::max(lc, maxl);
            }
            if (minl < 1) { if (!status) status = 4; continue; }
            if (minl < maxl) emit(G.idx(minl - 1, cx, cy), G.idx(maxl - 1, cx, cy));
        }
    }
    (void)L;
    return status;
}

}  // namespace

extern "C" {

int orc_flt_stage(const orc_grid* g, const orc_flt* dags, int32_t n_batches, const int32_t* batch_off,
                  const int32_t* ids, const int64_t* route_off, const int32_t* routes,
                  const int64_t* route2_off, int32_t* routes2, int32_t remove_phase_one,
                  int32_t* demand_half, int32_t* timestamp, int32_t* stamp,
                  double* total_wirelength, int64_t* total_vias, int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Grid G(g);
    const size_t cells = size_t(g->L) * g->X * g->Y;
    std::vector<float> wcost(cells), vcost(cells);
    std::vector<double> presum(cells);
    int status = 0;
    for (int b = 0; b < n_batches; ++b) {
        const int n = batch_off[b + 1] - batch_off[b];
        const int32_t* bid = ids + batch_off[b];
        if (remove_phase_one)  // flt.cuh:143-150
            commit_impl(g, n, bid, route_off, routes, ++*stamp, -1, demand_half, timestamp, total_wirelength,
                        total_vias, nullptr);
        const int32_t s = ++*stamp;  // flt.cuh:151
        orc_cost_full(g, demand_half, wcost.data(), vcost.data());  // refresh_cost: same values as incremental
        orc_presum(g, wcost.data(), presum.data());
#pragma omp parallel for schedule(dynamic, 4)
        for (int k = 0; k < n; ++k) {
            const int id = bid[k];
            const int rc = flt_net(G, dags, vcost.data(), presum.data(), id, routes2 + route2_off[id],
                                   route2_off[id + 1] - route2_off[id]);
            if (rc) {
#pragma omp critical
                if (!status) status = rc;
            }
        }
        commit_impl(g, n, bid, route2_off, routes2, s, 1, demand_half, timestamp, total_wirelength, total_vias,
                    nullptr);
    }
    return status;
}

}  // extern "C"


// ---------------------------------------------------------------------------
// Z-shape stage (pipeline_ggr.hpp:72-134, zshape.cuh:5-404,
// zshape_topology.hpp:7-57 and 249-290, demand.cuh:129-232).
namespace {

constexpr int kZInf = 1000000000;  // zshape.cuh:6

// 32-bit integer addition with wrap-around, as the device code computes it.
inline int zadd(int a, int b) { return static_cast<int>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b)); }

struct ZPlanes {
    int LAYER, N, D, L, X, Y;
    size_t NN, LNN;
    std::vector<int> map, prev;   // 6 and 16 planes of LAYER*N*N (pipeline_ggr.hpp:105-106)
    const double* presum;
    const float* vcost;
    int DIR;
    int pidx(int i, int x, int y) const { return int(i * NN + (((i & 1) ^ D) ? x * N + y : y * N + x)); }
    // WireCosts / ViaCosts (zshape.cuh:8-31): a plane index names (layer + 1, a, b).
    double wsum(int index) const {
        const int layer = index / int(NN) - 1;
        if (layer < 0 || layer >= L) return 0;
        const int a = index / N % N, b = index % N;
        const bool ay = ((layer & 1) ^ DIR) != 0;
        const int x = ay ? a : b, y = ay ? b : a;
        return presum[(size_t(layer) * X + x) * Y + y];
    }
    int vc(int index) const {
        const int layer = index / int(NN) - 1;
        if (layer < 0 || layer >= L) return kZInf;
        const int a = index / N % N, b = index % N;
        const bool ay = ((layer & 1) ^ DIR) != 0;
        const int x = ay ? a : b, y = ay ? b : a;
        return int(std::fmin(std::fmax(vcost[(size_t(layer) * X + x) * Y + y], 1.f), 1.e6f));
    }
    int wc(int a, int b) const { return int(std::fmin(std::fabs(wsum(a) - wsum(b)), double(kZInf / 2))); }
    int* M(int k) { return map.data() + k * LNN; }
    int* P(int k) { return prev.data() + k * LNN; }
    // viaSweep (zshape.cuh:42-61) on plane 4 at 2-D position (x, y).
    void via_sweep(int x, int y) {
        int* m = M(4);
        int* p = P(4);
        int* p5 = P(5);
        for (int i = 1; i < LAYER; ++i) {
            const int cur = int(i * NN + (((i & 1) ^ D) ? x * N + y : y * N + x));
            p5[cur] = cur;
        }
        for (int i = 2; i < LAYER; ++i) {
            const int cur = int(i * NN + (((i & 1) ^ D) ? x * N + y : y * N + x));
            const int last = int((i - 1) * NN + (((i & 1) ^ D) ? y * N + x : x * N + y));
            if (m[cur] > zadd(m[last], vc(last))) { m[cur] = zadd(m[last], vc(last)); p[cur] = p[last]; p5[cur] = last; }
        }
        for (int i = LAYER - 2; i >= 1; --i) {
            const int cur = int(i * NN + (((i & 1) ^ D) ? x * N + y : y * N + x));
            const int last = int((i + 1) * NN + (((i & 1) ^ D) ? y * N + x : x * N + y));
            if (m[cur] > zadd(m[last], vc(cur))) { m[cur] = zadd(m[last], vc(cur)); p[cur] = p[last]; p5[cur] = last; }
        }
    }
};

struct ZNode { int pos, minl, maxl, child[3]; };

// solve<4> (zshape.cuh:62-388) for one net, sequentially; `raw` receives the
// reference's route encoding: [count, (start, length | -1)...].
void zshape_net(ZPlanes& Z, const std::vector<ZNode>& nd, std::vector<int>& raw) {
    const int LAYER = Z.LAYER, N = Z.N, D = Z.D;
    raw.assign(1, 1);
    const int cnt = int(nd.size());
    int* map0 = Z.M(0);
    int* prev0 = Z.P(0);
    int* m4 = Z.M(4);
    int* p4 = Z.P(4);
    int* p5 = Z.P(5);
    int* m5 = Z.M(5);
    // reset_nodes (zshape.cuh:392-404).
    for (const auto& v : nd)
        for (int l = 0; l < LAYER; ++l)
            for (int plane = 0; plane < 4; ++plane) Z.M(plane)[Z.pidx(l, v.pos / N, v.pos % N)] = kZInf;
    for (int t = cnt - 1; t >= 0; --t) {
        const int tox = nd[t].pos / N, toy = nd[t].pos % N, minlayer = nd[t].minl, maxlayer = nd[t].maxl;
        for (int j = 1; j <= 3; ++j) {
            if (nd[t].child[j - 1] == -1) continue;
            int* mj = Z.M(j);
            int* pj = Z.P(j);
            int* p2j = Z.P(10 + j);
            const int cp = nd[nd[t].child[j - 1]].pos, fromx = cp / N, fromy = cp % N;
            const int minx = std::min(fromx, tox), maxx = std::max(fromx, tox);
            const int miny = std::min(fromy, toy), maxy = std::max(fromy, toy);
            if (fromx != tox && fromy != toy) {
                for (int a = minx; a <= maxx; ++a)
                    for (int i = 1; i < LAYER; ++i) {
                        if ((i & 1) ^ D) { m4[i * Z.NN + a * N + toy] = kZInf; m4[i * Z.NN + a * N + fromy] = kZInf; }
                        else { m4[i * Z.NN + toy * N + a] = kZInf; m4[i * Z.NN + fromy * N + a] = kZInf; }
                    }
                for (int b = miny; b <= maxy; ++b)
                    for (int i = 1; i < LAYER; ++i) {
                        if ((i & 1) ^ D) { m4[i * Z.NN + tox * N + b] = kZInf; m4[i * Z.NN + fromx * N + b] = kZInf; }
                        else { m4[i * Z.NN + b * N + tox] = kZInf; m4[i * Z.NN + b * N + fromx] = kZInf; }
                    }
                for (int i = 1; i < LAYER; ++i) {
                    if ((i & 1) ^ D) {
                        const int last = int(i * Z.NN + fromx * N + fromy);
                        for (int b = miny; b <= maxy; ++b) {
                            if (b == fromy) continue;
                            const int cur = int(i * Z.NN + fromx * N + b);
                            m4[cur] = zadd(map0[last], Z.wc(last, cur));
                            p4[cur] = last;
                        }
                    } else {
                        const int last = int(i * Z.NN + fromy * N + fromx);
                        for (int b = minx; b <= maxx; ++b) {
                            if (b == fromx) continue;
                            const int cur = int(i * Z.NN + fromy * N + b);
                            m4[cur] = zadd(map0[last], Z.wc(last, cur));
                            p4[cur] = last;
                        }
                    }
                }
                for (int b = miny; b <= maxy; ++b) if (b != fromy) Z.via_sweep(fromx, b);
                for (int b = minx; b <= maxx; ++b) if (b != fromx) Z.via_sweep(b, fromy);
                for (int i = 1; i < LAYER; ++i) {
                    if ((i & 1) ^ D) {
                        for (int b = minx; b <= maxx; ++b) {
                            const int last = int(i * Z.NN + b * N + fromy), cur = int(i * Z.NN + b * N + toy);
                            const int c = Z.wc(last, cur);
                            if (zadd(m4[last], c) < m4[cur]) { m4[cur] = zadd(m4[last], c); p4[cur] = p4[last]; }
                        }
                    } else {
                        for (int b = miny; b <= maxy; ++b) {
                            const int last = int(i * Z.NN + b * N + fromx), cur = int(i * Z.NN + b * N + tox);
                            const int c = Z.wc(last, cur);
                            if (zadd(m4[last], c) < m4[cur]) { m4[cur] = zadd(m4[last], c); p4[cur] = p4[last]; }
                        }
                    }
                }
                for (int b = miny; b <= maxy; ++b) if (b != toy) Z.via_sweep(tox, b);
                for (int b = minx; b <= maxx; ++b) if (b != tox) Z.via_sweep(b, toy);
                for (int i = 1; i < LAYER; ++i) {
                    if ((i & 1) ^ D) {
                        const int cur = int(i * Z.NN + tox * N + toy);
                        for (int b = miny; b <= maxy; ++b) {
                            if (b == toy) continue;
                            const int last = int(i * Z.NN + tox * N + b);
                            const int c = Z.wc(last, cur);
                            if (zadd(m4[last], c) < mj[cur]) { mj[cur] = zadd(m4[last], c); pj[cur] = p4[last]; p2j[cur] = p5[last]; }
                        }
                    } else {
                        const int cur = int(i * Z.NN + toy * N + tox);
                        for (int b = minx; b <= maxx; ++b) {
                            if (b == tox) continue;
                            const int last = int(i * Z.NN + toy * N + b);
                            const int c = Z.wc(last, cur);
                            if (zadd(m4[last], c) < mj[cur]) { mj[cur] = zadd(m4[last], c); pj[cur] = p4[last]; p2j[cur] = p5[last]; }
                        }
                    }
                }
            } else if (fromx == tox) {
                for (int i = 1; i < LAYER; ++i) {
                    if ((i & 1) ^ D) {
                        const int last = int(i * Z.NN + fromx * N + fromy), cur = int(i * Z.NN + tox * N + toy);
                        const int c = Z.wc(last, cur);
                        if (mj[cur] > zadd(map0[last], c)) { mj[cur] = zadd(map0[last], c); pj[cur] = last; }
                    } else {
                        mj[i * Z.NN + toy * N + tox] = kZInf;
                    }
                }
            } else if (fromy == toy) {
                for (int i = 1; i < LAYER; ++i) {
                    if ((!(i & 1)) ^ D) {
                        const int last = int(i * Z.NN + fromy * N + fromx), cur = int(i * Z.NN + toy * N + tox);
                        const int c = Z.wc(last, cur);
                        if (mj[cur] > zadd(map0[last], c)) { mj[cur] = zadd(map0[last], c); pj[cur] = last; }
                    } else {
                        mj[i * Z.NN + tox * N + toy] = kZInf;
                    }
                }
            }
        }
        // Layer-range DP at the node (zshape.cuh:241-267).
        for (int lower = 0; lower < LAYER; ++lower) {
            int viaSum = 0, minCost = kZInf, bestpos[3] = {0, 0, 0};
            int costs[3] = {nd[t].child[0] == -1 ? 0 : kZInf, nd[t].child[1] == -1 ? 0 : kZInf,
                            nd[t].child[2] == -1 ? 0 : kZInf};
            for (int upper = lower; upper < LAYER; ++upper) {
                const int idx = Z.pidx(upper, tox, toy);
                for (int j = 0; j < 3; ++j)
                    if (nd[t].child[j] != -1 && Z.M(j + 1)[idx] < costs[j]) { costs[j] = Z.M(j + 1)[idx]; bestpos[j] = upper; }
                if (1LL * costs[0] + costs[1] + costs[2] < minCost) minCost = costs[0] + costs[1] + costs[2];
                if (minlayer == -1 || (lower <= minlayer && maxlayer <= upper)) {
                    for (int i = lower; i <= upper; ++i) {
                        const int index = Z.pidx(i, tox, toy);
                        if (map0[index] > zadd(minCost, viaSum)) {
                            map0[index] = zadd(minCost, viaSum);
                            prev0[index] = (((lower * LAYER + upper) * LAYER + bestpos[2]) * LAYER + bestpos[1]) * LAYER + bestpos[0];
                        }
                    }
                }
                viaSum = zadd(viaSum, Z.vc(idx));
            }
        }
    }
    // Traceback (zshape.cuh:271-386).
    auto emit = [&](int a, int b) { raw.push_back(a); raw.push_back(b); raw[0] += 2; };
    int minTotal = kZInf;
    {
        const int x = nd[0].pos / N, y = nd[0].pos % N;
        for (int i = 0; i < LAYER; ++i) {
            const int idx = Z.pidx(i, x, y);
            if (map0[idx] < minTotal) { minTotal = map0[idx]; m5[nd[0].pos] = i; }
        }
    }
    if (minTotal == kZInf || minTotal < 0) { raw[0] = -1; return; }
    for (int t = 0; t < cnt; ++t) {
        const int x = nd[t].pos / N, y = nd[t].pos % N, layer = m5[nd[t].pos];
        const int idx = Z.pidx(layer, x, y);
        const int minl = prev0[idx] / LAYER / LAYER / LAYER / LAYER, maxl = prev0[idx] / LAYER / LAYER / LAYER % LAYER;
        for (int i = minl; i < maxl; ++i) emit(Z.pidx(i, x, y), -1);
        int bestpos = prev0[idx];
        for (int j = 0; j < 3; ++j) {
            if (nd[t].child[j] == -1) break;
            const int child = nd[nd[t].child[j]].pos;
            const int entrylayer = bestpos % LAYER, entry = Z.pidx(entrylayer, x, y);
            bestpos /= LAYER;
            const int last = Z.P(j + 1)[entry];
            const int lastlayer = last / int(Z.NN);
            int lastx = last / N % N, lasty = last % N;
            if ((!(lastlayer & 1)) ^ D) std::swap(lastx, lasty);
            if (lastx != x && lasty != y) {
                const int mid = Z.P(11 + j)[entry];
                const int midlayer = mid / int(Z.NN);
                int midx = mid / N % N, midy = mid % N;
                if ((!(midlayer & 1)) ^ D) std::swap(midx, midy);
                const int p1 = ((entrylayer & 1) ^ D) ? entry - y + midy : entry - x + midx;
                const int p3 = ((midlayer & 1) ^ D) ? mid - midy + lasty : mid - midx + lastx;
                const int p4 = ((lastlayer & 1) ^ D) ? last - lasty + midy : last - lastx + midx;
                if (entry != p1) emit(std::min(entry, p1), std::max(entry, p1) - std::min(entry, p1));
                if (p1 != mid)
                    for (int i = std::min(entrylayer, midlayer); i < std::max(entrylayer, midlayer); ++i) emit(Z.pidx(i, midx, midy), -1);
                if (mid != p3) emit(std::min(mid, p3), std::max(mid, p3) - std::min(mid, p3));
                if (p3 != p4) {
                    int tx = p3 / N % N, ty = p3 % N;
                    if ((!((p3 / int(Z.NN)) & 1)) ^ D) std::swap(tx, ty);
                    for (int i = std::min(midlayer, lastlayer); i < std::max(midlayer, lastlayer); ++i) emit(Z.pidx(i, tx, ty), -1);
                }
                if (p4 != last) emit(std::min(p4, last), std::max(p4, last) - std::min(p4, last));
            } else {
                emit(std::min(last, entry), std::max(last, entry) - std::min(last, entry));
            }
            m5[child] = lastlayer;
        }
    }
}

// convert_routes (zshape_topology.hpp:249-290).
int zshape_convert(const ZPlanes& Z, const std::vector<int>& src, int32_t* dst, int64_t cap) {
    int status = 0;
    const int n = Z.N, XY = Z.X * Z.Y;
    int out = 1;
    for (size_t p = 1; p + 1 < size_t(std::max(src[0], 0)); p += 2) {
        const int start = src[p], len = src[p + 1];
        const int layer = start / (n * n) - 1;
        const int a = start / n % n, b = start % n;
        const bool ay = ((layer & 1) ^ Z.DIR) != 0;
        const int x = ay ? a : b, y = ay ? b : a;
        if (layer < 0 || layer >= Z.L || x >= Z.X || y >= Z.Y) { status = 3; continue; }
        const int pos0 = layer * XY + x * Z.Y + y;
        int pos1 = pos0;
        if (len == -1) {
            if (layer + 1 >= Z.L) { status = 3; continue; }
            pos1 += XY;
        } else {
            const int end = start + len, ea = end / n % n, eb = end % n;
            const int ex = ay ? ea : eb, ey = ay ? eb : ea;
            if (ex >= Z.X || ey >= Z.Y) { status = 3; continue; }
            pos1 = layer * XY + ex * Z.Y + ey;
        }
        if (out + 1 < cap) { dst[out++] = pos0; dst[out++] = pos1; }
        else status = 1;
    }
    if (src[0] <= 0) status = 2;
    dst[0] = out;
    return status;
}

}  // namespace

extern "C" {

int orc_zshape_stage(const orc_grid* g, const orc_ztrees* trees, int32_t n_batches, const int32_t* batch_off,
                     const int32_t* ids, const int64_t* route_off, int32_t* routes, int32_t* demand_half,
                     int32_t* timestamp, int32_t* stamp, double* total_wirelength, int64_t* total_vias) {
    Grid G(g);
    ZPlanes Z;
    Z.L = g->L; Z.X = g->X; Z.Y = g->Y; Z.DIR = g->DIR;
    Z.LAYER = g->L + 1; Z.N = std::max(g->X, g->Y); Z.D = g->DIR ^ 1;
    Z.NN = size_t(Z.N) * Z.N; Z.LNN = Z.LAYER * Z.NN;
    Z.map.assign(6 * Z.LNN, 0);
    Z.prev.assign(16 * Z.LNN, 0);
    const size_t cells = size_t(g->L) * g->X * g->Y;
    std::vector<float> wcost(cells), vcost(cells);
    std::vector<double> presum(cells);
    Z.presum = presum.data();
    Z.vcost = vcost.data();
    int status = 0;
    std::vector<int> raw;
    std::vector<ZNode> nd;
    for (int b = 0; b < n_batches; ++b) {
        orc_cost_full(g, demand_half, wcost.data(), vcost.data());
        orc_presum(g, wcost.data(), presum.data());
        const int n = batch_off[b + 1] - batch_off[b];
        const int32_t* bid = ids + batch_off[b];
        for (int k = 0; k < n; ++k) {
            const int id = bid[k];
            const int nb = trees->node_off[id], cnt = trees->node_off[id + 1] - nb;
            nd.assign(cnt, ZNode{});
            for (int i = 0; i < cnt; ++i) {  // encode_batch (zshape_topology.hpp:100-116)
                const int c = trees->coord[nb + i], l = c / (g->X * g->Y), p2 = c % (g->X * g->Y);
                nd[i].pos = (p2 / g->Y) * Z.N + p2 % g->Y;
                nd[i].minl = nd[i].maxl = l < g->L ? l + 1 : -1;
                for (int j = 0; j < 3; ++j) nd[i].child[j] = trees->child[3 * (nb + i) + j];
            }
            if (cnt) zshape_net(Z, nd, raw);
            else raw.assign(1, 1);
            const int rc = zshape_convert(Z, raw, routes + route_off[id], route_off[id + 1] - route_off[id]);
            if (rc) status = rc;
        }
        const int32_t s = ++*stamp;
        commit_impl(g, n, bid, route_off, routes, s, 1, demand_half, timestamp, total_wirelength, total_vias, nullptr);
    }
    (void)G;
    return status;
}

int32_t orc_bbox_batches(int32_t X, int32_t Y, int32_t n, const int32_t* group, const int32_t* bbox,
                         int32_t max_batch, int32_t* ids, int32_t* off) {
    std::vector<int> pending(group, group + n);
    auto area = [&](int id) {
        return int64_t(bbox[4 * id + 1] - bbox[4 * id] + 1) * (bbox[4 * id + 3] - bbox[4 * id + 2] + 1);
    };
    std::sort(pending.begin(), pending.end(), [&](int l, int r) {
        return area(l) == area(r) ? l > r : area(l) > area(r);
    });
    std::vector<unsigned char> occupied(size_t(X) * Y, 0);
    int nb = 0, out = 0, routed = 0;
    off[0] = 0;
    while (routed < n) {
        std::fill(occupied.begin(), occupied.end(), 0);
        int count = 0;
        for (int& id : pending) {
            if (id < 0) continue;
            const int* bb = bbox + 4 * id;
            bool conflict = false;
            for (int x = bb[0]; x <= bb[1] && !conflict; ++x)
                for (int y = bb[2]; y <= bb[3]; ++y)
                    if (occupied[size_t(x) * Y + y]) { conflict = true; break; }
            if (conflict) continue;
            for (int x = bb[0]; x <= bb[1]; ++x)
                for (int y = bb[2]; y <= bb[3]; ++y) occupied[size_t(x) * Y + y] = 1;
            ids[out++] = id;
            id = -1;
            ++routed;
            if (++count == max_batch) break;
        }
        if (!count) break;
        off[++nb] = out;
    }
    return nb;
}

// construct_rsmt's geometry (preprocess.hpp:95-123) and Lshape_route's
// recursive depth-first flattening (lshape.cuh:85-98), net by net.
int orc_build_topology(int32_t X, int32_t Y, int32_t n, const int32_t* node_off, const int32_t* pos,
                       const int32_t* adj_off, const int32_t* adj, int32_t* nodes, int32_t* parents,
                       int32_t* point_off, int32_t* points, int32_t* hseg_off, int32_t* hsegs,
                       int32_t* vseg_off, int32_t* vsegs, int64_t* totals) {
    const int XY = X * Y;
    int np = 0, nh = 0, nv = 0;
    point_off[0] = hseg_off[0] = vseg_off[0] = 0;
    for (int id = 0; id < n; ++id) {
        const int base = node_off[id], N = node_off[id + 1] - base;
        // Adjacency must stay inside the net.
        for (int i = 0; i < N; ++i)
            for (int k = adj_off[base + i]; k < adj_off[base + i + 1]; ++k)
                if (adj[k] < 0 || adj[k] >= N) return -(id + 1);
        auto p2 = [&](int i) { return pos[base + i] % XY; };
        for (int i = 0; i < N; ++i) points[np++] = p2(i);
        for (int i = 0; i < N; ++i) {
            const int xi = p2(i) / Y, yi = p2(i) % Y;
            for (int k = adj_off[base + i]; k < adj_off[base + i + 1]; ++k) {
                const int j = adj[k];
                if (j >= i) continue;
                const int xj = p2(j) / Y, yj = p2(j) % Y;
                const int minx = std::min(xi, xj), maxx = std::max(xi, xj), miny = std::min(yi, yj),
                          maxy = std::max(yi, yj);
                if (xi != xj && yi != yj) {
                    hsegs[2 * nh] = minx * Y + miny; hsegs[2 * nh + 1] = maxx * Y + miny; ++nh;
                    hsegs[2 * nh] = minx * Y + maxy; hsegs[2 * nh + 1] = maxx * Y + maxy; ++nh;
                    vsegs[2 * nv] = minx * Y + miny; vsegs[2 * nv + 1] = minx * Y + maxy; ++nv;
                    vsegs[2 * nv] = maxx * Y + miny; vsegs[2 * nv + 1] = maxx * Y + maxy; ++nv;
                    points[np++] = xi * Y + yj;
                    points[np++] = xj * Y + yi;
                } else if (xi != xj) {
                    hsegs[2 * nh] = minx * Y + miny; hsegs[2 * nh + 1] = maxx * Y + miny; ++nh;
                    points[np++] = minx * Y + miny;
                    points[np++] = maxx * Y + miny;
                } else if (yi != yj) {
                    vsegs[2 * nv] = minx * Y + miny; vsegs[2 * nv + 1] = minx * Y + maxy; ++nv;
                    points[np++] = minx * Y + miny;
                    points[np++] = minx * Y + maxy;
                }
            }
        }
        point_off[id + 1] = np;
        hseg_off[id + 1] = nh;
        vseg_off[id + 1] = nv;
        // Recursive preorder; a node reached twice means the adjacency is
        // not a tree.
        int next = 0;
        bool bad = false;
        std::vector<char> seen(N, 0);
        std::function<void(int, int, int)> dfs = [&](int x, int par, int par_node) {
            if (bad || seen[x]) { bad = true; return; }
            seen[x] = 1;
            const int idx = next++;
            nodes[base + idx] = pos[base + x];
            parents[base + idx] = par_node;
            for (int k = adj_off[base + x]; k < adj_off[base + x + 1]; ++k)
                if (adj[k] != par) dfs(adj[k], x, idx);
        };
        if (N) dfs(0, -1, -1);
        if (bad || next != N) return -(id + 1);
    }
    totals[0] = np;
    totals[1] = nh;
    totals[2] = nv;
    return 0;
}

}  // extern "C"
