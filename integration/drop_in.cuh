// drop_in.cuh -- pieces shared by the drop-in drivers (grotor_grb.cu, the
// default pipeline; grotor_grb_ggr.cu, the GGR pipeline): error checks, the
// grid tables, the Steiner trees handed to grb_build_topology, the executor
// names and the device .out writer.  Included after the reference's pipeline
// headers, whose declarations (db::, cudb::, graph::, out_file) it uses.
#pragma once
#include <chrono>
#include <future>
#include <string>
#include <vector>

#include "grb.h"

namespace drop_in {

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
