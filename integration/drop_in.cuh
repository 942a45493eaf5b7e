// drop_in.cuh -- pieces shared by the drop-in drivers (grotor_grb.cu, the
// default pipeline; grotor_grb_ggr.cu, the GGR pipeline): error checks, the
// grid tables, the Steiner trees handed to grb_build_topology, the executor
// names and the device .out writer.  Included after the reference's pipeline
// headers, whose declarations (db::, cudb::, graph::, out_file) it uses.
#pragma once
#include <algorithm>
#include <chrono>
#include <memory>
#include <functional>
#include <future>
#include <string>
#include <vector>

#include "grb.h"

namespace drop_in {

// Host wall time of the program's phases (DROPIN_TIMING), from the clock
// that GROTOR_COMPLETE reads.
struct Phases {
    std::chrono::high_resolution_clock::time_point last = program_start;
    std::vector<std::pair<const char*, double>> ms;
    void mark(const char* name) {
        const auto now = std::chrono::high_resolution_clock::now();
        ms.emplace_back(name, std::chrono::duration<double, std::milli>(now - last).count());
        last = now;
    }
    void print() const {
        printf("DROPIN_TIMING");
        for (const auto& [name, v] : ms) printf(" %s_ms=%.3f", name, v);
        printf("\n");
    }
};
inline Phases phases;

// FLT nets whose widest DAG level holds more nodes than this go to a whole
// CTA (grb_set_flt_block_width; the library's default).
inline int flt_block_width = 32;

void check(int rc, grb_ctx* ctx, const char* what) {
    if (rc) throw std::runtime_error(std::string(what) + ": " + (ctx ? grb_last_error(ctx) : "error ") +
                                     " (code " + std::to_string(rc) + ")");
}

// The grid tables of build_cuda_database (preprocess.hpp:1625-1786).
struct Grid {
    std::vector<double> short_costs;
    std::vector<int32_t> xlen, ylen;
    std::vector<float> capacity;
    grb_grid g{};
};

Grid make_grid(const cudb::RouterState& state) {
    Grid G;
    const int L = state.device.L, X = state.device.X, Y = state.device.Y;
    for (int l = 0; l < L; ++l) G.short_costs.push_back(db::unit_length_short_costs[l + 1]);
    for (int x = 0; x + 1 < X; ++x) G.xlen.push_back(db::x_edge_len[x]);
    for (int y = 0; y + 1 < Y; ++y) G.ylen.push_back(db::y_edge_len[y]);
    G.capacity.resize(size_t(L) * X * Y);
    for (int l = 0; l < L; ++l)
        for (int x = 0; x < X; ++x)
            for (int y = 0; y < Y; ++y) G.capacity[(size_t(l) * X + x) * Y + y] = float(db::capacity[l + 1][x][y]);
    G.g.L = L;
    G.g.X = X;
    G.g.Y = Y;
    G.g.DIR = db::layers[1].dir;
    G.g.unit_length_wire_cost = db::unit_length_wire_cost;
    G.g.unit_via_cost = db::unit_via_cost;
    G.g.of_cost_scale = 1.0;  // router_state.hpp:37 on one GPU
    G.g.unit_length_short_costs = G.short_costs.data();
    G.g.x_edge_len = G.xlen.data();
    G.g.y_edge_len = G.ylen.data();
    G.g.capacity = G.capacity.data();
    return G;
}

// Every net's Steiner tree as FLUTE leaves it in net::rsmt (node positions
// with their layer, then each node's adjacency list; preprocess.hpp:72-93,
// 124-126) and its route words at the reference's own offsets
// (pin_cnt_sum_cpu * ROUTE_PER_PIN, router_state.hpp:31) -- all by net id.
// grb_build_topology turns them into the depth-first trees of Lshape_route
// (lshape.cuh:85-98) and the batching geometry of construct_rsmt
// (preprocess.hpp:95-123) on the device.
struct Trees {
    std::vector<int32_t> node_off{0}, pos, adj_off{0}, adj;
    std::vector<int64_t> route_off;
    grb_trees t{};
};

Trees flatten_trees(const cudb::RouterState& state) {
    Trees F;
    const auto& nets = state.nets;
    const int count = int(nets.size());
    for (int id = 0; id < count; ++id) {
        const auto& graph = nets[id].rsmt;
        const size_t size = graph.empty() ? 0 : graph.back().size();
        for (size_t i = 0; i < size; ++i) {
            F.pos.push_back(graph.back()[i]);
            F.adj.insert(F.adj.end(), graph[i].begin(), graph[i].end());
            F.adj_off.push_back(int32_t(F.adj.size()));
        }
        F.node_off.push_back(int32_t(F.pos.size()));
    }
    for (int id = 0; id <= count; ++id)
        F.route_off.push_back(int64_t(state.pin_cnt_sum_cpu[id]) * int64_t(state.device.ROUTE_PER_PIN));
    F.t.n = count;
    F.t.node_off = F.node_off.data();
    F.t.pos = F.pos.data();
    F.t.adj_off = F.adj_off.data();
    F.t.adj = F.adj.data();
    F.t.route_off = F.route_off.data();
    return F;
}

// Stage one: Lshape_route (lshape.cuh:21-197) with batching, cost refresh,
// DAG and commit on grotor_b200.  Leaves nets2route in the plan order, as
// the reference does; with `download`, the routes in state.routes_cpu.
void lshape_stage(cudb::RouterState& state, grb_ctx* ctx, std::vector<int>& nets2route, int32_t mode,
                  int64_t initial_vias, bool tail, bool download) {
    auto& nets = state.nets;
    const auto topology_start = std::chrono::steady_clock::now();
    // FLUTE only (construct_rsmt's rsmt_only form); the geometry and the
    // depth-first trees are built on the device.
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < int(nets2route.size()); ++i) nets[nets2route[i]].construct_rsmt(state, true);
    phases.mark("lshape_flute");
    Trees F = flatten_trees(state);
    check(grb_build_topology(ctx, &F.t), ctx, "grb_build_topology");
    phases.mark("lshape_topology");
    printf("TOPOLOGY_TIMING stage=lshape elapsed_ms=%.6f geometry_fused=0 executor=grotor_b200\n",
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - topology_start).count());
    std::sort(nets2route.begin(), nets2route.end(), [&](int l, int r) { return nets[l].hpwl > nets[r].hpwl; });
    check(grb_set_stats(ctx, 0.0, initial_vias), ctx, "grb_set_stats");
    int32_t nb = 0;
    check(grb_plan_batches(ctx, nets2route.data(), int32_t(nets2route.size()), 1000000, state.batch_sparsity_override,
                           mode == GRB_MODE_PERSISTENT ? GRB_MODE_PERSISTENT : GRB_MODE_PLAIN, nullptr, &nb),
          ctx, "grb_plan_batches");
    check(grb_set_stage_tail(ctx, tail ? (GRB_TAIL_RIPUP | GRB_TAIL_VIEW) : 0, 0), ctx, "grb_set_stage_tail");
    grb_stats st{};
    check(grb_lshape_stage(ctx, mode, &st), ctx, "grb_lshape_stage");
    phases.mark("lshape_stage");
    std::vector<int32_t> batch_off(nb + 1);
    int32_t n = 0, nb2 = 0;
    check(grb_get_plan(ctx, nets2route.data(), batch_off.data(), &n, &nb2), ctx, "grb_get_plan");
    if (download) {  // (the device writer reads the device's routes; a host copy is for host code)
        const size_t words = size_t(state.device.ROUTE_PER_PIN) * state.device.PIN_NUM + 1;
        state.routes_cpu.reset(new int[words]());
        check(grb_read_routes(ctx, state.routes_cpu.get()), ctx, "grb_read_routes");
    }
    printf("DAG_TIMING stage=lshape batch_index=-1 elapsed_ms=%.6f nets=%zu batches=%d executor=grotor_b200\n",
           st.dag_ms, nets2route.size(), nb);
    printf("BATCH_TIMING backend=grotor_b200 elapsed_ms=%.6f nets=%zu batches=%d used_for_routing=1\n",
           st.batching_ms, nets2route.size(), nb);
}

// prepare_detour_topology (flt.cuh:48-73) with the congestion view in host
// memory (from grb_read_stage_tail): the reference's host FLT DAG builder on
// nets2route, which it sorts by HPWL in place as the reference does.
void detour_prepare(cudb::RouterState& state, std::vector<int>& nets2route, const std::vector<unsigned char>& cong,
                    std::vector<float>& xsum, std::vector<float>& ysum) {
    auto& nets = state.nets;
    std::sort(nets2route.begin(), nets2route.end(), [&](int l, int r) { return nets[l].hpwl > nets[r].hpwl; });
    // The FLT builder keeps a net's stage-one RSMT segments (it runs with
    // construct_segments = false, flt.cuh:20); stage one built them on the
    // device, so the rerouted nets get them on the host here, from the same
    // trees (construct_rsmt is a pure function of net::rsmt and the pins).
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < int(nets2route.size()); ++i)
        if (!nets[nets2route[i]].rsmt.empty()) nets[nets2route[i]].construct_rsmt(state, false);
    std::unique_ptr<bool[]> view(new bool[cong.size()]);
    for (size_t i = 0; i < cong.size(); ++i) view[i] = cong[i] != 0;
    state.packing.congestionView_cpu = view.get();
    state.packing.congestionView_xsum_cpu = xsum.data();
    state.packing.congestionView_ysum_cpu = ysum.data();
    for (int id : nets2route) if (nets[id].rsmt.empty()) nets[id].construct_rsmt(state);
    state.flt_topology.begin(nets2route, nets.size(), 8);
    grotor::batching::prepare_geometry(state, nets2route, 8);
    Lshape_route_detour::multithreaded_processing(state, nets2route);
    state.packing.congestionView_cpu = nullptr;
    state.packing.congestionView_xsum_cpu = state.packing.congestionView_ysum_cpu = nullptr;
}

// The FLT executor -- route_prepared_topology's batching and batch loop
// (flt.cuh:75-182) -- on grotor_b200, once a DAG builder has filled
// state.flt_topology for nets2route (slot order) and set the nets' batching
// geometry (net::points and RSMT segments): the DAGs, the geometry of every
// net and phase-two route offsets (pins * words_per_pin words for each listed
// net, in id order) are uploaded, the nets batched (limit 300000) and the
// stage run (remove: rip up the listed nets' stage-one routes per batch).
// Nets flagged in `keep` get phase-two storage too (routes of an earlier
// stage that this one keeps); `before_stage` runs after the upload, to write
// them (grb_write_routes2).
struct FltRun {
    std::vector<int32_t> node_off{0}, coord, depth, children, parent_end, edge_off{0}, edge_parent, edge_slot;
    std::vector<int64_t> route2_off{0};
    grb_flt_dags d{};
    int32_t nb = 0;
    grb_stats st{};
};

FltRun flt_run(cudb::RouterState& state, grb_ctx* ctx, std::vector<int>& nets2route, int32_t mode, int remove,
               int64_t words_per_pin, const char* stage, const std::vector<uint8_t>* keep = nullptr,
               const std::function<void(FltRun&)>& before_stage = {}) {
    FltRun R;
    auto& nets = state.nets;
    const int count = int(nets.size());
    std::vector<int> slot_of(count, -1);
    for (size_t s = 0; s < nets2route.size(); ++s) slot_of[nets2route[s]] = int(s);
    std::vector<int32_t> point_off{0}, points, hseg_off{0}, hsegs, vseg_off{0}, vsegs;
    const auto& topo = state.flt_topology;
    for (int id = 0; id < count; ++id) {
        const int s = slot_of[id];
        if (s >= 0) {
            const auto& span = topo.spans[s];
            const auto& arena = topo.arenas[span.lane];
            for (int i = 0; i < span.nodes; ++i) {
                const auto& nd = arena.nodes[span.node_begin + i];
                R.coord.push_back(nd.coordinate);
                R.depth.push_back(nd.depth);
                R.children.push_back(nd.children);
                R.parent_end.push_back(nd.parent_end);
            }
            for (int i = 0; i < span.edges; ++i) {
                const auto& e = arena.edges[span.edge_begin + i];
                R.edge_parent.push_back(e.parent);
                R.edge_slot.push_back(e.source_slot);
            }
        }
        R.node_off.push_back(int32_t(R.coord.size()));
        R.edge_off.push_back(int32_t(R.edge_parent.size()));
        const auto& n = nets[id];
        if (s >= 0) {  // only the listed nets are batched: the others' ranges stay empty
            for (int p : n.points) points.push_back(p);
            for (const auto& sg : n.rsmt_h_segments) { hsegs.push_back(sg.first); hsegs.push_back(sg.second); }
            for (const auto& sg : n.rsmt_v_segments) { vsegs.push_back(sg.first); vsegs.push_back(sg.second); }
        }
        point_off.push_back(int32_t(points.size()));
        hseg_off.push_back(int32_t(hsegs.size() / 2));
        vseg_off.push_back(int32_t(vsegs.size() / 2));
        const bool stored = s >= 0 || (keep && (*keep)[id]);  // `keep`: storage for earlier stages' routes too
        const int64_t words = stored ? int64_t(n.pins.size()) * words_per_pin : 0;
        R.route2_off.push_back(R.route2_off.back() + words);
    }
    state.flt_topology.clear();
    phases.mark("flt_flatten");
    check(grb_upload_geometry(ctx, point_off.data(), points.data(), hseg_off.data(), hsegs.data(), vseg_off.data(),
                              vsegs.data()),
          ctx, "grb_upload_geometry");
    check(grb_plan_batches(ctx, nets2route.data(), int32_t(nets2route.size()), 300000, state.batch_sparsity_override,
                           mode == GRB_MODE_PERSISTENT ? GRB_MODE_PERSISTENT : GRB_MODE_PLAIN, nullptr, &R.nb),
          ctx, "grb_plan_batches (FLT)");
    R.d = grb_flt_dags{R.node_off.data(), R.coord.data(), R.depth.data(), R.children.data(), R.parent_end.data(),
                       R.edge_off.data(), R.edge_parent.data(), R.edge_slot.data(), R.route2_off.data()};
    check(grb_upload_flt(ctx, &R.d), ctx, "grb_upload_flt");
    check(grb_set_flt_block_width(ctx, flt_block_width), ctx, "grb_set_flt_block_width");
    if (before_stage) before_stage(R);
    phases.mark("flt_upload_plan");
    check(grb_flt_stage(ctx, remove, mode, &R.st), ctx, "grb_flt_stage");
    phases.mark("flt_stage");
    printf("DAG_TIMING stage=%s batch_index=-1 elapsed_ms=%.6f nets=%zu batches=%d executor=grotor_b200\n", stage,
           R.st.dag_ms, nets2route.size(), R.nb);
    printf("BATCH_TIMING stage=%s backend=grotor_b200 elapsed_ms=%.6f nets=%zu batches=%d used_for_routing=1\n", stage,
           R.st.batching_ms, nets2route.size(), R.nb);
    return R;
}

int32_t executor_mode(const std::string& name) {
    if (name == "persistent") return GRB_MODE_PERSISTENT;
    if (name == "plain") return GRB_MODE_PLAIN;
    if (name == "graph") return GRB_MODE_GRAPH;
    throw std::invalid_argument("--executor expects persistent, plain or graph");
}

// The .out writer (graph::output_nets, output.hpp:79-112) on the device: the
// ready records (collect_output_nets, output.hpp:16-26) are formatted by
// grb_format_out from the device's routes; a host task drains the text into
// the output file while the pipeline goes on (the reference's output task,
// pipeline.hpp:20-35), so the copy and the file write overlap the next stage.
struct Output {
    grb_ctx* ctx;
    std::future<int> task;
    double format_ms = 0, wait_ms = 0;

    static int sink(const char* data, int64_t bytes, void*) {
        return std::fwrite(data, 1, size_t(bytes), out_file) == size_t(bytes) ? 0 : 1;
    }
    void wait() {
        if (!task.valid()) return;
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = task.get();
        wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        check(rc, ctx, "grb_drain_out");
    }
    // Publish the ready nets (nets2output) as the next part of the file.
    void start(const cudb::RouterState& state) {
        wait();
        const auto t0 = std::chrono::steady_clock::now();
        auto ready = graph::collect_output_nets(std::move(nets2output));
        nets2output = {};
        std::vector<int64_t> name_off{0};
        std::string names;
        std::vector<int32_t> pin_off{0}, pins, extra_off{0}, extra, sub_off{0}, subnets;
        std::vector<uint8_t> phase2;
        for (const auto& r : ready) {
            names += r.name;
            name_off.push_back(int64_t(names.size()));
            pins.insert(pins.end(), r.pins.begin(), r.pins.end());
            pin_off.push_back(int32_t(pins.size()));
            extra.insert(extra.end(), r.extra_routes.begin(), r.extra_routes.end());
            extra_off.push_back(int32_t(extra.size()));
            for (int id : r.subnets) {
                subnets.push_back(id);
                phase2.push_back(state.ripup_flag_cpu[id] != 0);
            }
            sub_off.push_back(int32_t(subnets.size()));
        }
        grb_out_records rec{int32_t(ready.size()), name_off.data(), names.data(), pin_off.data(), pins.data(),
                            extra_off.data(), extra.data(), sub_off.data(), subnets.data(), phase2.data()};
        int64_t bytes = 0;
        check(grb_format_out(ctx, &rec, &bytes), ctx, "grb_format_out");
        format_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        grb_ctx* c = ctx;
        task = std::async(std::launch::async, [c] { return grb_drain_out(c, &Output::sink, nullptr); });
    }
};

}  // namespace drop_in
