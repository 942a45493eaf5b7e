// synth.cpp -- seeded synthetic designs and routing topology (host side).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/grb_synth.h"

struct grb_design {
    grb_synth_params p{};
    std::string error;
    int L = 0, X = 0, Y = 0, DIR = 1;
    std::vector<double> short_costs;
    std::vector<int32_t> xlen, ylen;
    std::vector<float> capacity;         // routing layers [L][X][Y]
    std::vector<float> cap_layer0;       // CAP layer 0 (metal1), written to CAP files only
    std::vector<int32_t> pin_off, pins;  // CAP-layer pin ids per net
    // topology
    std::vector<int32_t> node_off, nodes, parents, point_off, points, hseg_off, hsegs, vseg_off, vsegs;
    std::vector<int64_t> route_off;
    std::vector<int32_t> hpwl, original, pin_count;
    // Z-shape encoding of the same trees (built on request)
    std::vector<int32_t> z_node_off, z_coord, z_child;
};

namespace {

// splitmix64 seeding + xoshiro-style generator through std::mt19937_64.
struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t seed) : g(seed) {}
    double uniform() { return (g() >> 11) * (1.0 / 9007199254740992.0); }
    int range(int lo, int hi) { return lo + int(g() % uint64_t(hi - lo + 1)); }
    double normal() {
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2 * M_PI * u2);
    }
};

uint64_t mix(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

int draw_pins(const grb_synth_params& p, Rng& r) {
    int n;
    if (p.pin_model == 1) {
        const double u = std::max(r.uniform(), 1e-12);
        const double lomax = std::pow(u, -1.0 / p.pareto_alpha) - 1.0;
        n = 2 + int(std::min(lomax, 1e6));
    } else {
        if (r.uniform() < p.two_pin_frac) n = 2;
        else {
            n = 3;
            while (n < p.max_pins && r.uniform() >= p.geo_p) ++n;
        }
    }
    return std::min(n, p.max_pins);
}

int draw_side(const grb_synth_params& p, Rng& r, int limit, bool big) {
    double s;
    if (p.bbox_model == 1) s = std::exp(r.uniform() * std::log(double(std::max(p.bbox_max, 1))));
    else if (big) s = r.range(p.big_lo, p.big_hi);
    else s = std::exp(std::log(p.bbox_median) + p.bbox_sigma * r.normal());
    int v = int(std::lround(s));
    return std::max(1, std::min(v, limit));
}

inline int manhattan(int a, int b, int Y) { return std::abs(a / Y - b / Y) + std::abs(a % Y - b % Y); }

// Rectilinear MST over 2-D cell ids (Prim, O(n^2)); returns parent per node
// (rooted at node 0).
std::vector<int> rmst(const std::vector<int>& pos, int Y) {
    const int n = int(pos.size());
    std::vector<int> par(n, -1), best(n, INT32_MAX);
    std::vector<char> in(n, 0);
    best[0] = 0;
    for (int it = 0; it < n; ++it) {
        int u = -1;
        for (int i = 0; i < n; ++i)
            if (!in[i] && (u < 0 || best[i] < best[u])) u = i;
        in[u] = 1;
        for (int v = 0; v < n; ++v)
            if (!in[v]) {
                const int d = manhattan(pos[u], pos[v], Y);
                if (d < best[v]) { best[v] = d; par[v] = u; }
            }
    }
    return par;
}

struct Tree {
    std::vector<int> pos;                 // 2-D ids
    std::vector<int> layer;               // routing layer, L for Steiner
    std::vector<std::vector<int>> adj;
};

int med3(int a, int b, int c) { return std::max(std::min(a, b), std::min(std::max(a, b), c)); }

// Greedy median Steiner points on an MST: repeatedly replace the pair of edges
// (u,a), (u,b) with the largest saving by a Steiner point at the component-wise
// median of u, a, b.
void add_steiner(Tree& t, int L, int Y) {
    const int pins = int(t.pos.size());
    for (int guard = 0; guard < pins; ++guard) {
        int bu = -1, ba = -1, bb = -1, bs = -1, gain = 0;
        for (int u = 0; u < int(t.pos.size()); ++u) {
            const auto& nb = t.adj[u];
            for (size_t i = 0; i < nb.size(); ++i)
                for (size_t j = i + 1; j < nb.size(); ++j) {
                    const int a = nb[i], b = nb[j];
                    const int ux = t.pos[u] / Y, uy = t.pos[u] % Y, ax = t.pos[a] / Y, ay = t.pos[a] % Y,
                              bx = t.pos[b] / Y, by = t.pos[b] % Y;
                    const int s = med3(ux, ax, bx) * Y + med3(uy, ay, by);
                    const int g = manhattan(t.pos[u], t.pos[a], Y) + manhattan(t.pos[u], t.pos[b], Y) -
                                  manhattan(t.pos[u], s, Y) - manhattan(s, t.pos[a], Y) - manhattan(s, t.pos[b], Y);
                    if (g > gain) { gain = g; bu = u; ba = a; bb = b; bs = s; }
                }
        }
        if (gain <= 0) break;
        if (std::find(t.pos.begin(), t.pos.end(), bs) != t.pos.end()) break;
        const int s = int(t.pos.size());
        t.pos.push_back(bs);
        t.layer.push_back(L);
        t.adj.emplace_back();
        auto drop = [&](int x, int y) { auto& v = t.adj[x]; v.erase(std::find(v.begin(), v.end(), y)); };
        drop(bu, ba); drop(ba, bu); drop(bu, bb); drop(bb, bu);
        for (int v : {bu, ba, bb}) { t.adj[s].push_back(v); t.adj[v].push_back(s); }
    }
}

struct Subnet {
    std::vector<int> pos, layer;  // 2-D ids and routing layers of the pins
    int original;
};

// Split a net above `cap` pins into connected subnets of at most `cap` pins that
// share one pin with their neighbour (the shared pin keeps the union connected).
void split_net(const std::vector<int>& pos, const std::vector<int>& layer, int cap, int Y, int original,
               std::vector<Subnet>& out) {
    const int n = int(pos.size());
    if (n <= cap) { out.push_back({pos, layer, original}); return; }
    const std::vector<int> par = rmst(pos, Y);
    std::vector<std::vector<int>> kids(n);
    for (int v = 1; v < n; ++v) kids[par[v]].push_back(v);
    std::vector<int> post;
    std::vector<int> stack{0};
    std::vector<int> order;
    while (!stack.empty()) {
        const int v = stack.back(); stack.pop_back();
        order.push_back(v);
        for (int k : kids[v]) stack.push_back(k);
    }
    std::reverse(order.begin(), order.end());  // children before parents
    std::vector<std::vector<int>> open(n);      // open cluster members of each node
    for (int v : order) {
        std::vector<int> cl{v};
        std::vector<int> ks = kids[v];
        for (int k : ks) cl.insert(cl.end(), open[k].begin(), open[k].end());
        while (int(cl.size()) > cap - 1) {
            // Cut off the largest open child cluster with v as its shared pin.
            int big = -1;
            for (int k : ks)
                if (!open[k].empty() && (big < 0 || open[k].size() > open[big].size())) big = k;
            if (big < 0) break;
            Subnet s;
            s.original = original;
            for (int m : open[big]) { s.pos.push_back(pos[m]); s.layer.push_back(layer[m]); }
            s.pos.push_back(pos[v]); s.layer.push_back(layer[v]);
            out.push_back(std::move(s));
            std::unordered_set<int> gone(open[big].begin(), open[big].end());
            std::vector<int> keep;
            for (int m : cl) if (!gone.count(m)) keep.push_back(m);
            cl.swap(keep);
            open[big].clear();
        }
        open[v] = cl;
        for (int k : ks) open[k].clear();
    }
    if (open[0].size() >= 1) {
        Subnet s;
        s.original = original;
        for (int m : open[0]) { s.pos.push_back(pos[m]); s.layer.push_back(layer[m]); }
        if (s.pos.size() >= 2) out.push_back(std::move(s));
    }
}

struct NetTopo {
    std::vector<int> nodes, parents, points, hsegs, vsegs;
    int hpwl = 0;
};

// Tree, DFS order and batching geometry of one subnet, with the node order and
// point/segment rules of net::construct_rsmt (preprocess.hpp:88-130) and the
// DFS of lshape.cuh:85-103.
NetTopo build_tree(const Subnet& s, int L, int X, int Y) {
    Tree t;
    t.pos = s.pos;
    t.layer = s.layer;
    t.adj.assign(t.pos.size(), {});
    const std::vector<int> par = rmst(t.pos, Y);
    for (int v = 1; v < int(par.size()); ++v) { t.adj[v].push_back(par[v]); t.adj[par[v]].push_back(v); }
    add_steiner(t, L, Y);
    // Sort nodes by 2-D id (the reference sorts FLUTE nodes) and remap.
    const int n = int(t.pos.size());
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return t.pos[a] < t.pos[b]; });
    std::vector<int> rank(n);
    for (int i = 0; i < n; ++i) rank[idx[i]] = i;
    std::vector<std::vector<int>> adj(n);
    std::vector<int> pos(n), lay(n);
    for (int i = 0; i < n; ++i) {
        pos[i] = t.pos[idx[i]];
        lay[i] = t.layer[idx[i]];
        for (int v : t.adj[idx[i]]) adj[i].push_back(rank[v]);
    }
    NetTopo o;
    int minx = X, maxx = 0, miny = Y, maxy = 0;
    for (size_t k = 0; k < s.pos.size(); ++k) {
        minx = std::min(minx, s.pos[k] / Y); maxx = std::max(maxx, s.pos[k] / Y);
        miny = std::min(miny, s.pos[k] % Y); maxy = std::max(maxy, s.pos[k] % Y);
    }
    o.hpwl = maxx - minx + maxy - miny;
    // Batching geometry.
    o.points = pos;
    for (int i = 0; i < n; ++i) {
        const int xi = pos[i] / Y, yi = pos[i] % Y;
        for (int j : adj[i]) {
            if (j >= i) continue;
            const int xj = pos[j] / Y, yj = pos[j] % Y;
            const int mnx = std::min(xi, xj), mxx = std::max(xi, xj), mny = std::min(yi, yj), mxy = std::max(yi, yj);
            if (xi != xj && yi != yj) {
                o.hsegs.insert(o.hsegs.end(), {mnx * Y + mny, mxx * Y + mny, mnx * Y + mxy, mxx * Y + mxy});
                o.vsegs.insert(o.vsegs.end(), {mnx * Y + mny, mnx * Y + mxy, mxx * Y + mny, mxx * Y + mxy});
                o.points.push_back(xi * Y + yj);
                o.points.push_back(xj * Y + yi);
            } else if (xi != xj) {
                o.hsegs.insert(o.hsegs.end(), {mnx * Y + mny, mxx * Y + mny});
                o.points.push_back(mnx * Y + mny);
                o.points.push_back(mxx * Y + mny);
            } else if (yi != yj) {
                o.vsegs.insert(o.vsegs.end(), {mnx * Y + mny, mnx * Y + mxy});
                o.points.push_back(mnx * Y + mny);
                o.points.push_back(mnx * Y + mxy);
            }
        }
    }
    // DFS from node 0 (neighbours in adjacency order).
    std::vector<std::pair<int, int>> st{{0, -1}};
    std::vector<char> seen(n, 0);
    std::vector<int> dfs_index(n, -1);
    while (!st.empty()) {
        const auto [v, parent_dfs] = st.back();
        st.pop_back();
        if (seen[v]) continue;
        seen[v] = 1;
        const int me = int(o.nodes.size());
        dfs_index[v] = me;
        o.nodes.push_back(lay[v] * X * Y + pos[v]);
        o.parents.push_back(parent_dfs);
        for (auto it = adj[v].rbegin(); it != adj[v].rend(); ++it)
            if (!seen[*it]) st.push_back({*it, me});
    }
    return o;
}

}  // namespace

extern "C" {

grb_design* grb_synth_generate(const grb_synth_params* pp) {
    auto* d = new grb_design;
    if (!pp || pp->X < 2 || pp->Y < 2 || pp->cap_layers < 2 || pp->cap_layers > 11 || pp->n_nets < 0) {
        d->error = "invalid synthesis parameters";
        return d;
    }
    const grb_synth_params& p = *pp;
    d->p = p;
    d->L = p.cap_layers - 1;
    d->X = p.X;
    d->Y = p.Y;
    d->DIR = 1;  // CAP layer 1 (first routing layer) runs along y
    const size_t XY = size_t(p.X) * p.Y;
    d->short_costs.assign(d->L, p.overflow_weight);
    d->xlen.assign(p.X - 1, 1);
    d->ylen.assign(p.Y - 1, 1);
    d->capacity.resize(size_t(d->L) * XY);
    d->cap_layer0.resize(XY);
    Rng rc(mix(p.seed * 2 + 1));
    std::vector<char> blocked(XY, 0);
    for (size_t i = 0; i < XY; ++i) blocked[i] = p.blockage > 0 && rc.uniform() < p.blockage;
    for (size_t i = 0; i < XY; ++i) d->cap_layer0[i] = float(rc.range(p.cap_lo, p.cap_hi));
    for (int l = 0; l < d->L; ++l)
        for (size_t i = 0; i < XY; ++i) {
            const int v = rc.range(p.cap_lo, p.cap_hi);
            d->capacity[l * XY + i] = blocked[i] ? 0.f : float(v);
        }
    // Nets: each net draws from its own stream, so any subset is reproducible.
    d->pin_off.assign(1, 0);
    std::vector<int> cells;
    for (int k = 0; k < p.n_nets; ++k) {
        Rng r(mix(p.seed * 1000003ull + uint64_t(k) * 7919ull + 17));
        int np = draw_pins(p, r);
        const bool big = p.bbox_model == 0 && r.uniform() < p.big_frac;
        int w = draw_side(p, r, p.X, big), h = draw_side(p, r, p.Y, big);
        while (size_t(w) * h < size_t(np)) {
            if (w < p.X) ++w;
            if (size_t(w) * h < size_t(np) && h < p.Y) ++h;
            if (w == p.X && h == p.Y) break;
        }
        np = int(std::min<size_t>(np, size_t(w) * h));
        const int x0 = r.range(0, p.X - w), y0 = r.range(0, p.Y - h);
        std::unordered_set<int> used;
        cells.clear();
        while (int(cells.size()) < np) {
            const int x = x0 + r.range(0, w - 1), y = y0 + r.range(0, h - 1);
            const int c = x * p.Y + y;
            if (used.insert(c).second) cells.push_back(c);
        }
        for (int c : cells) {
            const int l = r.range(0, std::max(p.pin_cap_layers, 1) - 1);
            d->pins.push_back(int32_t(l * int(XY) + c));
        }
        d->pin_off.push_back(int32_t(d->pins.size()));
    }
    return d;
}

void grb_design_free(grb_design* d) { delete d; }
const char* grb_design_error(const grb_design* d) { return d ? d->error.c_str() : "null design"; }

int grb_design_grid(const grb_design* d, grb_grid* g) {
    if (!d || !g || !d->error.empty()) return GRB_EINVAL;
    g->L = d->L; g->X = d->X; g->Y = d->Y; g->DIR = d->DIR;
    g->unit_length_wire_cost = d->p.unit_wire;
    g->unit_via_cost = d->p.unit_via;
    g->of_cost_scale = 1.0;
    g->unit_length_short_costs = d->short_costs.data();
    g->x_edge_len = d->xlen.data();
    g->y_edge_len = d->ylen.data();
    g->capacity = d->capacity.data();
    return GRB_OK;
}

int grb_design_write(const grb_design* d, const char* cap_path, const char* net_path) {
    if (!d || !d->error.empty()) return GRB_EINVAL;
    const int CL = d->L + 1, X = d->X, Y = d->Y;
    const size_t XY = size_t(X) * Y;
    FILE* f = std::fopen(cap_path, "w");
    if (!f) return GRB_EINVAL;
    std::fprintf(f, "%d %d %d\n%.8g %.8g", CL, X, Y, d->p.unit_wire, d->p.unit_via);
    std::fprintf(f, " %.8g", d->p.overflow_weight);  // CAP layer 0
    for (int l = 0; l < d->L; ++l) std::fprintf(f, " %.8g", d->short_costs[l]);
    std::fprintf(f, "\n");
    for (int i = 0; i < X - 1; ++i) std::fprintf(f, "%d ", d->xlen[i]);
    std::fprintf(f, "\n");
    for (int i = 0; i < Y - 1; ++i) std::fprintf(f, "%d ", d->ylen[i]);
    std::fprintf(f, "\n");
    for (int l = 0; l < CL; ++l) {
        // CAP layer l direction: layer 1 carries the routing direction DIR.
        const int dir = ((l - 1) & 1) ^ d->DIR;
        std::fprintf(f, "metal%d %d 1\n", l + 1, l == 0 ? (d->DIR ^ 1) : dir);
        std::string line;
        for (int y = 0; y < Y; ++y) {
            line.clear();
            for (int x = 0; x < X; ++x) {
                const float c = l == 0 ? d->cap_layer0[size_t(x) * Y + y] : d->capacity[(l - 1) * XY + size_t(x) * Y + y];
                line += std::to_string(int(c));
                line += ' ';
            }
            line += '\n';
            std::fputs(line.c_str(), f);
        }
    }
    std::fclose(f);
    FILE* g = std::fopen(net_path, "w");
    if (!g) return GRB_EINVAL;
    const int n = int(d->pin_off.size()) - 1;
    for (int k = 0; k < n; ++k) {
        std::fprintf(g, "net%d\n(\n", k);
        for (int q = d->pin_off[k]; q < d->pin_off[k + 1]; ++q) {
            const int p = d->pins[q], l = int(p / XY), r = int(p % XY);
            std::fprintf(g, "[(%d, %d, %d)]\n", l, r / Y, r % Y);
        }
        std::fprintf(g, ")\n");
    }
    std::fclose(g);
    return GRB_OK;
}

int grb_design_build_topology(grb_design* d, int32_t cap, int32_t threads) {
    if (!d || !d->error.empty() || cap < 2) return GRB_EINVAL;
    const int L = d->L, X = d->X, Y = d->Y;
    const int XY = X * Y;
    const int n = int(d->pin_off.size()) - 1;
    // Split into subnets (1-pin nets need no routing, preprocess.hpp:1474).
    std::vector<std::vector<Subnet>> parts(n);
    int T = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    auto run = [&](auto&& body, int count) {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t)
            pool.emplace_back([&, t] { for (int k = t; k < count; k += T) body(k); });
        for (auto& th : pool) th.join();
    };
    run([&](int k) {
        std::vector<int> pos, lay;
        for (int q = d->pin_off[k]; q < d->pin_off[k + 1]; ++q) {
            const int p = d->pins[q], l = p / XY;
            pos.push_back(p % XY);
            lay.push_back(l >= 1 ? l - 1 : 0);  // CAP layer l -> routing layer l-1 (layer 0 stays 0)
        }
        if (pos.size() >= 2) split_net(pos, lay, cap, Y, k, parts[k]);
    }, n);
    std::vector<Subnet> subs;
    for (auto& v : parts) for (auto& s : v) subs.push_back(std::move(s));
    parts.clear();
    const int m = int(subs.size());
    std::vector<NetTopo> topo(m);
    run([&](int k) { topo[k] = build_tree(subs[k], L, X, Y); }, m);
    d->node_off.assign(1, 0); d->point_off.assign(1, 0); d->hseg_off.assign(1, 0); d->vseg_off.assign(1, 0);
    d->route_off.assign(1, 0);
    d->nodes.clear(); d->parents.clear(); d->points.clear(); d->hsegs.clear(); d->vsegs.clear();
    d->hpwl.assign(m, 0); d->original.assign(m, 0); d->pin_count.assign(m, 0);
    for (int k = 0; k < m; ++k) {
        const auto& t = topo[k];
        d->nodes.insert(d->nodes.end(), t.nodes.begin(), t.nodes.end());
        d->parents.insert(d->parents.end(), t.parents.begin(), t.parents.end());
        d->points.insert(d->points.end(), t.points.begin(), t.points.end());
        d->hsegs.insert(d->hsegs.end(), t.hsegs.begin(), t.hsegs.end());
        d->vsegs.insert(d->vsegs.end(), t.vsegs.begin(), t.vsegs.end());
        d->node_off.push_back(int32_t(d->nodes.size()));
        d->point_off.push_back(int32_t(d->points.size()));
        d->hseg_off.push_back(int32_t(d->hsegs.size() / 2));
        d->vseg_off.push_back(int32_t(d->vsegs.size() / 2));
        // A node emits at most one via pair and one L (3 pairs): 8 words.
        d->route_off.push_back(d->route_off.back() + 1 + 8 * int64_t(t.nodes.size()));
        d->hpwl[k] = t.hpwl;
        d->original[k] = subs[k].original;
        d->pin_count[k] = int(subs[k].pos.size());
    }
    return GRB_OK;
}

int grb_design_nets(const grb_design* d, grb_nets* o) {
    if (!d || !o || d->node_off.empty()) return GRB_EINVAL;
    o->n = int32_t(d->node_off.size()) - 1;
    o->node_off = d->node_off.data(); o->nodes = d->nodes.data(); o->parents = d->parents.data();
    o->route_off = d->route_off.data();
    o->point_off = d->point_off.data(); o->points = d->points.data();
    o->hseg_off = d->hseg_off.data(); o->hsegs = d->hsegs.data();
    o->vseg_off = d->vseg_off.data(); o->vsegs = d->vsegs.data();
    return GRB_OK;
}

int grb_design_subnet_info(const grb_design* d, const int32_t** hpwl, const int32_t** original, const int32_t** pc) {
    if (!d || d->node_off.empty()) return GRB_EINVAL;
    if (hpwl) *hpwl = d->hpwl.data();
    if (original) *original = d->original.data();
    if (pc) *pc = d->pin_count.data();
    return GRB_OK;
}

int grb_design_order(const grb_design* d, int32_t* order) {
    if (!d || !order || d->node_off.empty()) return GRB_EINVAL;
    const int m = int(d->hpwl.size());
    std::iota(order, order + m, 0);
    std::stable_sort(order, order + m, [&](int a, int b) { return d->hpwl[a] > d->hpwl[b]; });
    return GRB_OK;
}

int grb_design_zshape_trees(grb_design* d, const int32_t** node_off, const int32_t** coord, const int32_t** child) {
    if (!d || d->node_off.empty()) return GRB_EINVAL;
    if (d->z_node_off.empty()) {
        const int m = int(d->node_off.size()) - 1;
        d->z_node_off.assign(1, 0);
        d->z_coord.reserve(d->nodes.size());
        d->z_child.reserve(3 * d->nodes.size());
        std::vector<std::vector<int>> adj, kids;
        std::vector<int> crd, order, pre, stack;
        for (int k = 0; k < m; ++k) {
            const int a = d->node_off[k], n = d->node_off[k + 1] - a;
            adj.assign(n, {});
            for (int i = 1; i < n; ++i) {
                const int p = d->parents[a + i];
                adj[i].push_back(p);
                adj[p].push_back(i);
            }
            for (auto& v : adj) std::sort(v.begin(), v.end());
            int root = 0;  // the first leaf, as zshape_topology.hpp:80-82
            for (int i = 0; i < n; ++i) if (adj[i].size() == 1) { root = i; break; }
            // Rooted children lists.  A node with more than three children
            // hands the extra ones to the nearest node of its first child's
            // subtree that has room (the Z-shape DP keeps one plane cell per
            // 2-D position, so no two tree nodes may share a position).
            kids.assign(n, {});
            crd.assign(n, 0);
            for (int i = 0; i < n; ++i) crd[i] = d->nodes[a + i];
            std::vector<int> par(n, -1);
            stack.assign(1, root);
            par[root] = root;
            while (!stack.empty()) {
                const int v = stack.back(); stack.pop_back();
                for (int w : adj[v]) if (par[w] == -1) { par[w] = v; kids[v].push_back(w); stack.push_back(w); }
            }
            for (int v = 0; v < n; ++v) {
                while (kids[v].size() > 3) {
                    const int extra = kids[v].back();
                    kids[v].pop_back();
                    std::vector<int> queue{kids[v][0]};
                    for (size_t h = 0; h < queue.size(); ++h) {
                        const int w = queue[h];
                        if (kids[w].size() < 3) { kids[w].push_back(extra); break; }
                        for (int x : kids[w]) queue.push_back(x);
                    }
                }
            }
            const int nn = int(kids.size());
            order.clear(); pre.assign(nn, -1); stack.assign(1, root);
            while (!stack.empty()) {
                const int v = stack.back(); stack.pop_back();
                pre[v] = int(order.size());
                order.push_back(v);
                for (auto it = kids[v].rbegin(); it != kids[v].rend(); ++it) stack.push_back(*it);
            }
            for (int v : order) {
                d->z_coord.push_back(crd[v]);
                for (int j = 0; j < 3; ++j) d->z_child.push_back(j < int(kids[v].size()) ? pre[kids[v][j]] : -1);
            }
            d->z_node_off.push_back(int32_t(d->z_coord.size()));
        }
    }
    if (node_off) *node_off = d->z_node_off.data();
    if (coord) *coord = d->z_coord.data();
    if (child) *child = d->z_child.data();
    return GRB_OK;
}

int grb_design_pins(const grb_design* d, const int32_t** pin_off, const int32_t** pins, int32_t* n) {
    if (!d || !d->error.empty()) return GRB_EINVAL;
    if (pin_off) *pin_off = d->pin_off.data();
    if (pins) *pins = d->pins.data();
    if (n) *n = int32_t(d->pin_off.size()) - 1;
    return GRB_OK;
}

}  // extern "C"
