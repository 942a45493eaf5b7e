// ref_harness.cu -- drives the reference router's own code on a CAP/NET design
// and dumps its intermediate and final results for the parity tests.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/ref.mk from the reference sources
// where they lie (include path only, nothing copied); the binary lands in
// oracle/_ref/.  Modes:
//   topo  <cap> <net> <dir> <lut>   CPU: subnets, FLUTE trees (DFS order as in
//                                   Lshape_route), batching geometry, HPWL order,
//                                   CPU first-fit batches, grid tables.
//   route <cap> <net> <dir> <lut> <out>
//                                   GPU: the reference L-shape stage
//                                   (build_cuda_database, Lshape_route), routes,
//                                   demand, statistics, refreshed cost tables and
//                                   the .out file written by the reference writer.
//   snap  <cap> <net> <dir> <lut> <k>
//                                   GPU: reference per-batch kernels over the dumped
//                                   plan; cost tables before batch k, routes after.
//   batch <dir> <limit> <sparsity>  CPU: time generate_batches_rsmt on a dumped
//                                   geometry (X, Y, order, points, segments).
//   flt   <cap> <net> <dir> <lut>   GPU: the reference default pipeline up to and
//                                   through its FLT stage (pipeline.hpp:86-137):
//                                   L-shape, congestion view, rip-up, the host FLT
//                                   DAG builder; dumps the DAGs, the FLT batching
//                                   geometry and batches and the state before the
//                                   stage, runs route_prepared_topology and dumps
//                                   phase-two routes, demand and statistics.
//   zshape <cap> <net> <dir> <lut>  GPU, GGR build only (ref_harness_ggr, compiled with
//                                   GROTOR_GGR_ROUTING): the reference Z-shape
//                                   pipeline (pipeline_ggr.hpp:8-144) -- order,
//                                   first-fit groups, bbox batches, the encoded
//                                   trees and net boxes, then routes, demand and
//                                   statistics after the stage, before the host
//                                   post-processing (:145-151).
//   write <cap> <net> <dir> <lut> <routes> <out>
//                                   CPU: write a .out with the reference writer from
//                                   route words produced elsewhere (nets published
//                                   in the plan order <dir>/ids.i32 when present).
// Every array is written as raw little-endian data, <dir>/<name>.<i32|i64|f32|f64>.
#include "pipeline.hpp"
#ifdef GROTOR_GGR_ROUTING
#include "pipeline_ggr.hpp"
#endif

#include <filesystem>
#include <fstream>
#include <numeric>

namespace {

template <class T>
void dump(const std::string& dir, const std::string& name, const T* data, size_t count) {
    const char* ext = std::is_same_v<T, int> ? ".i32" : std::is_same_v<T, long long> ? ".i64"
                    : std::is_same_v<T, float> ? ".f32" : ".f64";
    std::ofstream f(dir + "/" + name + ext, std::ios::binary);
    f.write(reinterpret_cast<const char*>(data), sizeof(T) * count);
}
template <class T>
void dump(const std::string& dir, const std::string& name, const std::vector<T>& v) { dump(dir, name, v.data(), v.size()); }

template <class T>
std::vector<T> load(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot read " + path);
    const size_t bytes = f.tellg();
    f.seekg(0);
    std::vector<T> v(bytes / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), bytes);
    return v;
}

void read_design(const std::string& cap, const std::string& net, const std::string& lut) {
    std::string c = cap, n = net;
    db::read(c.data(), n.data());
    const auto cwd = std::filesystem::current_path();
    std::filesystem::current_path(lut);
    flute::readLUT();
    std::filesystem::current_path(cwd);
}

void dump_grid(const std::string& dir, cudb::RouterState& state) {
    const int L = state.device.L, X = state.device.X, Y = state.device.Y;
    std::vector<int> meta{L, X, Y, state.device.DIR};
    dump(dir, "meta", meta);
    std::vector<double> sc(L), units{db::unit_length_wire_cost, db::unit_via_cost};
    for (int l = 0; l < L; ++l) sc[l] = db::unit_length_short_costs[l + 1];
    dump(dir, "short_costs", sc);
    dump(dir, "unit_costs", units);
    dump(dir, "x_edge_len", db::x_edge_len);
    dump(dir, "y_edge_len", db::y_edge_len);
    std::vector<float> cap(size_t(L) * X * Y);
    for (int l = 0; l < L; ++l)
        for (int x = 0; x < X; ++x)
            for (int y = 0; y < Y; ++y) cap[(size_t(l) * X + x) * Y + y] = float(db::capacity[l + 1][x][y]);
    dump(dir, "capacity", cap);
}

int run_topo(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut) {
    read_design(cap, net, lut);
    cudb::RouterState state;
    state.batch_sparsity_override = 1;
    cudb::prepare_routing_nets(state);
    auto& nets = state.nets;
    const int n = nets.size();
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < n; ++i) nets[i].construct_rsmt(state, false);  // lshape.cuh:33-36
    std::vector<int> order = all;
    std::sort(order.begin(), order.end(), [&](int l, int r) { return nets[l].hpwl > nets[r].hpwl; });  // lshape.cuh:53-55
    std::vector<int> sorted = order;
    auto batches = cudb::generate_batches_rsmt(state, sorted, 1000000, 1);
    std::vector<int> batch_of(n, -1), pos(n);
    for (int i = 0; i < n; ++i) pos[order[i]] = i;
    for (size_t b = 0; b < batches.size(); ++b)
        for (int id : batches[b]) batch_of[pos[id]] = int(b);
    std::reverse(batches.begin(), batches.end());  // lshape.cuh:70
    std::vector<int> ids, batch_off{0};
    for (auto& b : batches) { ids.insert(ids.end(), b.begin(), b.end()); batch_off.push_back(ids.size()); }
    // Per-net DFS flattening exactly as lshape.cuh:85-103.
    std::vector<int> node_off{0}, nodes, parents, point_off{0}, points, hseg_off{0}, hsegs, vseg_off{0}, vsegs;
    std::vector<int> hpwl(n), original(n), pin_count(n);
    // The trees themselves (net::rsmt after construct_rsmt: node positions
    // with their layer, then each node's adjacency list), for the topology
    // construction's parity.
    std::vector<int> rsmt_pos, rsmt_adj_off{0}, rsmt_adj;
    for (int id = 0; id < n; ++id) {
        auto& graph = nets[id].rsmt;
        for (size_t i = 0; i + 1 < graph.size(); ++i) {
            rsmt_pos.push_back(graph.back()[i]);
            rsmt_adj.insert(rsmt_adj.end(), graph[i].begin(), graph[i].end());
            rsmt_adj_off.push_back(rsmt_adj.size());
        }
        const size_t base = nodes.size();
        nodes.resize(base + graph.back().size());
        parents.resize(base + graph.back().size());
        int cnt = 0;
        std::function<void(int, int, int)> dfs = [&](int x, int par, int par_node) {
            const int idx = cnt++;
            nodes[base + idx] = graph.back()[x];
            parents[base + idx] = par_node;
            for (int e : graph[x]) if (e != par) dfs(e, x, idx);
        };
        dfs(0, -1, -1);
        node_off.push_back(nodes.size());
        for (int p : nets[id].points) points.push_back(p);
        point_off.push_back(points.size());
        for (auto& s : nets[id].rsmt_h_segments) { hsegs.push_back(s.first); hsegs.push_back(s.second); }
        hseg_off.push_back(hsegs.size() / 2);
        for (auto& s : nets[id].rsmt_v_segments) { vsegs.push_back(s.first); vsegs.push_back(s.second); }
        vseg_off.push_back(vsegs.size() / 2);
        hpwl[id] = nets[id].hpwl;
        original[id] = nets[id].original_net_id;
        pin_count[id] = nets[id].pins.size();
    }
    dump_grid(dir, state);
    dump(dir, "pin_acc_num", state.pin_cnt_sum_cpu);
    // Initial via statistic: one via per metal1 pin (preprocess.hpp:1716-1718).
    std::vector<int> pin_vias{0};
    for (auto& dbnet : db::nets)
        for (int pin : dbnet.pins) pin_vias[0] += pin < state.device.X * state.device.Y;
    dump(dir, "pin_vias", pin_vias);
    dump(dir, "node_off", node_off); dump(dir, "nodes", nodes); dump(dir, "parents", parents);
    dump(dir, "rsmt_pos", rsmt_pos); dump(dir, "rsmt_adj_off", rsmt_adj_off); dump(dir, "rsmt_adj", rsmt_adj);
    dump(dir, "point_off", point_off); dump(dir, "points", points);
    dump(dir, "hseg_off", hseg_off); dump(dir, "hsegs", hsegs);
    dump(dir, "vseg_off", vseg_off); dump(dir, "vsegs", vsegs);
    dump(dir, "hpwl", hpwl); dump(dir, "original", original); dump(dir, "pin_count", pin_count);
    dump(dir, "order", order); dump(dir, "batch_of", batch_of);
    dump(dir, "ids", ids); dump(dir, "batch_off", batch_off);
    printf("REF_TOPO nets=%d batches=%zu nodes=%zu\n", n, batches.size(), nodes.size());
    return 0;
}

int run_route(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut,
              const std::string& out) {
    read_design(cap, net, lut);
    out_file = fopen(out.c_str(), "w");
    if (!out_file) throw std::runtime_error("cannot open " + out);
    setvbuf(out_file, nullptr, _IONBF, 0);
    std::vector<int> ids, words;
    {
        cudb::RouterState state;
        state.batch_sparsity_override = 1;
        state.report_score = false;
        // pipeline.hpp:36-67, stage one only.
        cudb::build_cuda_database(state);
        graph::initialize_incremental_cost(state);
        auto& view = state.device;
        for (int i = 0; i < int(db::nets.size()); ++i)
            if (db::nets[i].pins.size() == 1) nets2output.push(i);
        grotor::cuda_check(cudaFuncSetAttribute(graph::compute_presum,
                   cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(double) * view.XY), "prefix shared memory");
        std::vector<int> all(state.nets.size());
        std::iota(all.begin(), all.end(), 0);
        Lshape_route::Lshape_route(state, all);
        grotor::cuda_check(cudaDeviceSynchronize(), "L-shape stage");
        state.download_routes(false);
        const size_t cells = size_t(view.L) * view.X * view.Y;
        std::vector<float> demand(cells), wcost(cells), vcost(cells);
        std::vector<double> presum(cells);
        cudaMemcpy(demand.data(), view.demand, cells * 4, cudaMemcpyDeviceToHost);
        cudb::RoutingStatistics stats;
        cudaMemcpy(&stats, view.statistics, sizeof(stats), cudaMemcpyDeviceToHost);
        graph::refresh_cost(state);  // costs of the final demand
        grotor::cuda_check(cudaDeviceSynchronize(), "final refresh");
        cudaMemcpy(wcost.data(), view.wcost, cells * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(vcost.data(), view.vcost, cells * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(presum.data(), view.presum, cells * 8, cudaMemcpyDeviceToHost);
        const size_t count = view.ROUTE_PER_PIN * view.PIN_NUM + 1;
        dump(dir, "ref_routes", state.routes_cpu.get(), count);
        dump(dir, "ref_demand", demand); dump(dir, "ref_wcost", wcost); dump(dir, "ref_vcost", vcost);
        dump(dir, "ref_presum", presum);
        std::vector<double> st{stats.total_wirelength, double(stats.total_via_count)};
        dump(dir, "ref_stats", st);
        graph::finish_nets(state, all);  // pipeline.hpp:71-77
        auto records = graph::collect_output_nets(std::move(nets2output));
        nets2output = {};
        graph::output_nets(state, std::move(records));
        state.release_workspaces();
    }
    fclose(out_file);
    out_file = nullptr;
    printf("REF_ROUTE done\n");
    return 0;
}

// GPU: the reference's per-batch kernels (graph::refresh_cost,
// Lshape_route_warp, graph::commit_batch_demand) driven in the order of
// lshape.cuh:153-179 over the dumped plan; before batch `snap` the cost tables
// are saved, after it the batch's routes.  Lets the CPU tests feed the
// reference's own tables to the oracle's DP.
int run_snap(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut,
             int snap) {
    read_design(cap, net, lut);
    cudb::RouterState state;
    state.batch_sparsity_override = 1;
    cudb::build_cuda_database(state);
    graph::initialize_incremental_cost(state);
    auto& view = state.device;
    const auto ids = load<int>(dir + "/ids.i32"), batch_off = load<int>(dir + "/batch_off.i32");
    const auto node_off_id = load<int>(dir + "/node_off.i32"), nodes_id = load<int>(dir + "/nodes.i32");
    const auto parents_id = load<int>(dir + "/parents.i32");
    const int n = ids.size(), nb = batch_off.size() - 1, L = view.L;
    if (snap < 0) snap += nb;
    // Flatten per execution position (lshape.cuh:80-103 layout).
    std::vector<int> node_cnt_sum{0}, nodes, par_nodes;
    for (int id : ids) {
        for (int k = node_off_id[id]; k < node_off_id[id + 1]; ++k) {
            nodes.push_back(nodes_id[k]);
            par_nodes.push_back(parents_id[k]);
        }
        node_cnt_sum.push_back(nodes.size());
    }
    int max_nodes = 0;
    for (int b = 0; b < nb; ++b) max_nodes = std::max(max_nodes, node_cnt_sum[batch_off[b + 1]] - node_cnt_sum[batch_off[b]]);
    int *d_ncs, *d_nodes, *d_par, *d_from, *d_range;
    double* d_dist;
    cudaMalloc(&d_ncs, node_cnt_sum.size() * 4); cudaMalloc(&d_nodes, nodes.size() * 4);
    cudaMalloc(&d_par, nodes.size() * 4); cudaMalloc(&d_range, nodes.size() * 4);
    cudaMalloc(&d_dist, size_t(max_nodes) * L * L * 8); cudaMalloc(&d_from, size_t(max_nodes) * L * L * 4);
    cudaMemcpy(d_ncs, node_cnt_sum.data(), node_cnt_sum.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_nodes, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_par, par_nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(view.net_ids, ids.data(), n * 4, cudaMemcpyHostToDevice);
    grotor::cuda_check(cudaFuncSetAttribute(graph::compute_presum,
               cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(double) * view.XY), "prefix shared memory");
    auto routing_view = state.device;
    routing_view.pre_demand = nullptr;
    const size_t cells = size_t(L) * view.X * view.Y;
    for (int b = 0; b <= snap; ++b) {
        ++state.global_timestamp;
        graph::refresh_cost(state);
        if (b == snap) {
            grotor::cuda_check(cudaDeviceSynchronize(), "snapshot");
            std::vector<float> wcost(cells), vcost(cells), demand(cells);
            std::vector<double> presum(cells);
            cudaMemcpy(wcost.data(), view.wcost, cells * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(vcost.data(), view.vcost, cells * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(presum.data(), view.presum, cells * 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(demand.data(), view.demand, cells * 4, cudaMemcpyDeviceToHost);
            dump(dir, "snap_wcost", wcost); dump(dir, "snap_vcost", vcost);
            dump(dir, "snap_presum", presum); dump(dir, "snap_demand", demand);
        }
        const int cnt = batch_off[b + 1] - batch_off[b];
        Lshape_route::Lshape_route_warp<<<(cnt + 3) / 4, 128>>>(routing_view, cnt, batch_off[b], d_ncs, d_nodes, d_par,
                                                               d_dist, d_from, d_range, state.global_timestamp);
        graph::commit_batch_demand(state.device, cnt, batch_off[b], state.global_timestamp);
    }
    grotor::cuda_check(cudaDeviceSynchronize(), "snap stage");
    state.download_routes(false);
    dump(dir, "snap_routes", state.routes_cpu.get(), view.ROUTE_PER_PIN * view.PIN_NUM + 1);
    std::vector<int> meta{snap};
    dump(dir, "snap_batch", meta);
    printf("REF_SNAP batch=%d of %d\n", snap, nb);
    return 0;
}

int run_flt(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut) {
    read_design(cap, net, lut);
    cudb::RouterState state;
    state.batch_sparsity_override = 1;
    state.report_score = false;
    cudb::build_cuda_database(state);
    graph::initialize_incremental_cost(state);
    auto& view = state.device;
    grotor::cuda_check(cudaFuncSetAttribute(graph::compute_presum,
               cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(double) * view.XY), "prefix shared memory");
    grotor::cuda_check(cudaFuncSetAttribute(graph::compute_presum_general,
               cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(int) * view.XY), "demand shared memory");
    std::vector<int> all(state.nets.size());
    std::iota(all.begin(), all.end(), 0);
    Lshape_route::Lshape_route(state, all);
    grotor::cuda_check(cudaDeviceSynchronize(), "L-shape stage");
    const size_t cells = size_t(view.L) * view.X * view.Y;
    auto dump_state = [&](const std::string& tag) {
        std::vector<float> demand(cells);
        cudaMemcpy(demand.data(), view.demand, cells * 4, cudaMemcpyDeviceToHost);
        cudb::RoutingStatistics stats;
        cudaMemcpy(&stats, view.statistics, sizeof(stats), cudaMemcpyDeviceToHost);
        dump(dir, tag + "_demand", demand);
        std::vector<double> st{stats.total_wirelength, double(stats.total_via_count), double(state.global_timestamp)};
        dump(dir, tag + "_stats", st);
    };
    dump_state("flt_before");
    // pipeline.hpp:86-106: mode, congestion view, rip-up, phase-two offsets.
    if (state.nets.size() > 5000000) mode = 1;
    if (state.nets.size() > 20000000) mode = 2;
    graph::extract_congestionView<<<BLOCK_NUM(view.X * view.Y), THREAD_NUM>>>(view);
    graph::extract_congestionView_xsum<<<view.Y, THREAD_NUM, sizeof(float) * view.X>>>(view);
    graph::extract_congestionView_ysum<<<view.X, THREAD_NUM, sizeof(float) * view.Y>>>(view);
    {
        // The congestion view the host FLT builder reads (congestion.cuh:60-112).
        const size_t xy = size_t(view.X) * view.Y;
        std::vector<unsigned char> cong(xy);
        std::vector<float> xsum(xy), ysum(xy);
        grotor::cuda_check(cudaMemcpy(cong.data(), view.congestion, xy, cudaMemcpyDeviceToHost), "congestion");
        grotor::cuda_check(cudaMemcpy(xsum.data(), view.congestion_xsum, 4 * xy, cudaMemcpyDeviceToHost), "xsum");
        grotor::cuda_check(cudaMemcpy(ysum.data(), view.congestion_ysum, 4 * xy, cudaMemcpyDeviceToHost), "ysum");
        std::vector<int> cong_i(cong.begin(), cong.end());
        dump(dir, "flt_congestion", cong_i);
        dump(dir, "flt_xsum", xsum);
        dump(dir, "flt_ysum", ysum);
    }
    auto overflow_nets = graph::ripup(state, 0);
    dump(dir, "flt_of_nets", overflow_nets.first);
    int pin_count = 0;
    for (auto net_id : overflow_nets.first) {
        state.pin_cnt_sum_phase2_cpu[net_id] = pin_count;
        pin_count += state.nets[net_id].pins.size();
        state.ripup_flag_cpu[net_id] = 1;
    }
    view.PIN_NUM_PHASE2 = pin_count;
    state.memory.allocate(&view.routes_phase2, (view.ROUTE_PER_PIN_PHASE2 * pin_count + 1) * sizeof(int));
    cudaMemcpy(view.ripup_flag, state.ripup_flag_cpu.data(), (1 + view.NET_NUM) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(view.pin_acc_num_phase2, state.pin_cnt_sum_phase2_cpu.data(), (1 + view.NET_NUM) * sizeof(int),
               cudaMemcpyHostToDevice);
    dump(dir, "flt_pin_acc2", state.pin_cnt_sum_phase2_cpu);
    std::vector<int> nets2route = overflow_nets.first;
    // flt.cuh:48-73: sort by HPWL, host DAG builder, batching geometry.
    Lshape_route_detour::prepare_detour_topology(state, nets2route);
    dump(dir, "flt_nets", nets2route);
    auto& topo = state.flt_topology;
    std::vector<int> node_off{0}, coord, depth, children, parent_end, edge_off{0}, edge_parent, edge_slot;
    std::vector<int> point_off{0}, points, hseg_off{0}, hsegs, vseg_off{0}, vsegs;
    for (size_t slot = 0; slot < nets2route.size(); ++slot) {
        const auto& span = topo.spans[slot];
        const auto& arena = topo.arenas[span.lane];
        for (int i = 0; i < span.nodes; ++i) {
            const auto& nd = arena.nodes[span.node_begin + i];
            coord.push_back(nd.coordinate); depth.push_back(nd.depth);
            children.push_back(nd.children); parent_end.push_back(nd.parent_end);
        }
        for (int i = 0; i < span.edges; ++i) {
            const auto& e = arena.edges[span.edge_begin + i];
            edge_parent.push_back(e.parent); edge_slot.push_back(e.source_slot);
        }
        node_off.push_back(coord.size()); edge_off.push_back(edge_parent.size());
        const auto& n = state.nets[nets2route[slot]];
        for (int p : n.points) points.push_back(p);
        point_off.push_back(points.size());
        for (auto& sg : n.rsmt_h_segments) { hsegs.push_back(sg.first); hsegs.push_back(sg.second); }
        hseg_off.push_back(hsegs.size() / 2);
        for (auto& sg : n.rsmt_v_segments) { vsegs.push_back(sg.first); vsegs.push_back(sg.second); }
        vseg_off.push_back(vsegs.size() / 2);
    }
    dump(dir, "flt_node_off", node_off); dump(dir, "flt_coord", coord); dump(dir, "flt_depth", depth);
    dump(dir, "flt_children", children); dump(dir, "flt_parent_end", parent_end);
    dump(dir, "flt_edge_off", edge_off); dump(dir, "flt_edge_parent", edge_parent); dump(dir, "flt_edge_slot", edge_slot);
    dump(dir, "flt_point_off", point_off); dump(dir, "flt_points", points);
    dump(dir, "flt_hseg_off", hseg_off); dump(dir, "flt_hsegs", hsegs);
    dump(dir, "flt_vseg_off", vseg_off); dump(dir, "flt_vsegs", vsegs);
    // The stage's batches (flt.cuh:92, executed in reverse, flt_topology.hpp:101).
    std::vector<int> sorted = nets2route;
    auto batches = cudb::generate_batches_rsmt(state, sorted, 300000, state.batch_sparsity_override);
    std::vector<int> batch_ids, batch_off{0};
    for (auto it = batches.rbegin(); it != batches.rend(); ++it) {
        if (it->empty()) continue;
        batch_ids.insert(batch_ids.end(), it->begin(), it->end());
        batch_off.push_back(batch_ids.size());
    }
    dump(dir, "flt_batch_ids", batch_ids); dump(dir, "flt_batch_off", batch_off);
    Lshape_route_detour::route_prepared_topology(state, nets2route, "detour", true);
    grotor::cuda_check(cudaDeviceSynchronize(), "FLT stage");
    dump_state("flt_after");
    state.download_routes(true);
    dump(dir, "flt_routes2", state.routes_phase2_cpu.get(), view.ROUTE_PER_PIN_PHASE2 * view.PIN_NUM_PHASE2 + 1);
    state.download_routes(false);
    dump(dir, "flt_routes1", state.routes_cpu.get(), view.ROUTE_PER_PIN * view.PIN_NUM + 1);
    printf("REF_FLT nets=%zu batches=%zu nodes=%zu edges=%zu\n", nets2route.size(), batch_off.size() - 1,
           coord.size(), edge_parent.size());
    state.release_workspaces();
    return 0;
}

#ifdef GROTOR_GGR_ROUTING
int run_zshape(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut) {
    read_design(cap, net, lut);
    cudb::RouterState state;
    state.batch_sparsity_override = 1;
    state.report_score = false;
    // pipeline_ggr.hpp:9-71.
    state.device.ROUTE_PER_PIN = 256;
    cudb::build_cuda_database(state);
    graph::initialize_incremental_cost(state);
    auto& view = state.device;
    grotor::cuda_check(cudaFuncSetAttribute(graph::compute_presum,
               cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(double) * view.XY), "prefix shared memory");
    const int n = std::max(view.X, view.Y), layers = view.L + 1;
    const size_t grid = size_t(layers) * n * n;
    std::vector<int> order(state.nets.size());
    std::iota(order.begin(), order.end(), 0);
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < int(order.size()); ++i) state.nets[i].construct_rsmt(state, false);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return state.nets[a].hpwl == state.nets[b].hpwl ? a > b : state.nets[a].hpwl > state.nets[b].hpwl;
    });
    auto groups = cudb::generate_batches_rsmt(state, order, 1000000, 1);
    std::vector<std::vector<int>> batches;
    for (const auto& group : groups) {
        auto refined = grotor::zshape::generate_bbox_batches(group, state.nets, view.X, view.Y);
        for (auto& batch : refined) batches.emplace_back(std::move(batch));
    }
    std::reverse(batches.begin(), batches.end());
    std::vector<int> group_ids, group_off{0}, zb_ids, zb_off{0};
    for (auto& g : groups) { group_ids.insert(group_ids.end(), g.begin(), g.end()); group_off.push_back(group_ids.size()); }
    for (auto& b : batches) { zb_ids.insert(zb_ids.end(), b.begin(), b.end()); zb_off.push_back(zb_ids.size()); }
    dump_grid(dir, state);
    dump(dir, "pin_acc_num", state.pin_cnt_sum_cpu);
    std::vector<int> pin_vias{0};  // initial via statistic (preprocess.hpp:1716-1718)
    for (auto& dbnet : db::nets)
        for (int pin : dbnet.pins) pin_vias[0] += pin < view.X * view.Y;
    dump(dir, "pin_vias", pin_vias);
    dump(dir, "z_order", order); dump(dir, "z_group_ids", group_ids); dump(dir, "z_group_off", group_off);
    dump(dir, "z_batch_ids", zb_ids); dump(dir, "z_batch_off", zb_off);
    // Per-net trees in the encoding of zshape::encode_batch (zshape_topology.hpp:59-121),
    // with 3-D coordinates, and the net boxes used by generate_bbox_batches.
    std::vector<int> node_off{0}, coord, child, bbox;
    std::vector<int> zero_offsets(state.nets.size(), 0);
    for (int id = 0; id < int(state.nets.size()); ++id) {
        const auto& nt = state.nets[id];
        bbox.push_back(nt.minx); bbox.push_back(nt.maxx); bbox.push_back(nt.miny); bbox.push_back(nt.maxy);
        auto enc = grotor::zshape::encode_batch({id}, state.nets, zero_offsets, view.X, view.Y, view.L);
        const int* rec = enc.points.data() + enc.points[0];
        const int cnt = rec[1];
        // Recover each preorder node's 3-D coordinate from the tree (the
        // encoding keeps only its 2-D position and pin layer range).
        const auto& graph = nt.rsmt;
        const int node_count = int(graph.size()) - 1;
        int root = 0;
        for (int i = 0; i < node_count; ++i) if (graph[i].size() == 1) { root = i; break; }
        std::vector<int> ord, parent(node_count, -1), stack{root};
        while (!stack.empty()) {
            const int v = stack.back(); stack.pop_back(); ord.push_back(v);
            for (auto it = graph[v].rbegin(); it != graph[v].rend(); ++it) {
                if (*it == parent[v]) continue;
                parent[*it] = v; stack.push_back(*it);
            }
        }
        for (int k = 0; k < cnt; ++k) {
            coord.push_back(graph.back()[ord[k]]);
            for (int j = 0; j < 3; ++j) child.push_back(rec[2 + 6 * k + 3 + j] < 0 ? -1 : rec[2 + 6 * k + 3 + j] / 6);
        }
        node_off.push_back(coord.size());
    }
    dump(dir, "z_node_off", node_off); dump(dir, "z_coord", coord); dump(dir, "z_child", child); dump(dir, "z_bbox", bbox);
    // pipeline_ggr.hpp:72-134: the batch loop, in the reference's structure.
    struct Span { size_t points, gbpoints, offsets, ids; int count, point_count, gb_count, raw_words; };
    std::vector<Span> spans;
    std::vector<int> points, gbpoints, offsets, ids, route_offsets(order.size());
    size_t max_points = 1, max_gb = 1, max_raw = 1;
    for (const auto& batch : batches) {
        int raw_words = 0;
        const size_t offset_begin = offsets.size();
        for (int id : batch) {
            route_offsets[id] = raw_words;
            offsets.push_back(raw_words);
            raw_words += int(state.nets[id].pins.size()) * 256;
        }
        auto encoded = grotor::zshape::encode_batch(batch, state.nets, route_offsets, view.X, view.Y, view.L);
        spans.push_back({points.size(), gbpoints.size(), offset_begin, ids.size(), int(batch.size()),
            int(encoded.points.size()), int(encoded.gbpoints.size()), raw_words});
        points.insert(points.end(), encoded.points.begin(), encoded.points.end());
        gbpoints.insert(gbpoints.end(), encoded.gbpoints.begin(), encoded.gbpoints.end());
        ids.insert(ids.end(), batch.begin(), batch.end());
        max_points = std::max(max_points, encoded.points.size());
        max_gb = std::max(max_gb, encoded.gbpoints.size());
        max_raw = std::max(max_raw, size_t(raw_words));
    }
    grotor::DeviceMemory memory;
    int *map = nullptr, *prev = nullptr, *raw = nullptr, *d_points = nullptr, *d_gb = nullptr, *d_offsets = nullptr, *error = nullptr;
    memory.allocate(&map, 6 * grid * sizeof(int));
    memory.allocate(&prev, 16 * grid * sizeof(int));
    memory.allocate(&raw, max_raw * sizeof(int));
    memory.allocate(&d_points, max_points * sizeof(int));
    memory.allocate(&d_gb, max_gb * sizeof(int));
    memory.allocate(&d_offsets, 251 * sizeof(int));
    memory.allocate(&error, sizeof(int));
    cudaMemset(error, 0, sizeof(int));
    for (const auto& batch : spans) {
        graph::refresh_cost(state);
        cudaMemcpy(d_points, points.data() + batch.points, batch.point_count * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(d_gb, gbpoints.data() + batch.gbpoints, batch.gb_count * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(d_offsets, offsets.data() + batch.offsets, batch.count * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(view.net_ids, ids.data() + batch.ids, batch.count * 4, cudaMemcpyHostToDevice);
        grotor::zshape::reset_nodes<<<batch.count, 128>>>(map, d_points, layers, n, view.DIR ^ 1, batch.count);
        grotor::zshape::solve<4><<<(batch.count + 3) / 4, 128>>>(map, d_points, {view, n}, {view, n}, prev,
            prev + 10 * grid, raw, d_gb, nullptr, layers, n, view.DIR ^ 1, batch.count);
        grotor::zshape::convert_routes<<<BLOCK_NUM(batch.count), THREAD_NUM>>>(batch.count, view.net_ids,
            d_offsets, raw, n, view.L, view.X, view.Y, view.DIR, view.ROUTE_PER_PIN, view.pin_acc_num, view.routes, error);
        const int stamp = ++state.global_timestamp;
        graph::commit_wire_demand<<<BLOCK_NUM(batch.count), THREAD_NUM>>>(view, batch.count, 0, stamp);
        graph::commit_via_demand<<<BLOCK_NUM(batch.count), THREAD_NUM>>>(view, batch.count, 0, stamp);
    }
    grotor::cuda_check(cudaDeviceSynchronize(), "Z-shape stage");
    int status = 0;
    cudaMemcpy(&status, error, sizeof(int), cudaMemcpyDeviceToHost);
    const size_t cells = size_t(view.L) * view.X * view.Y;
    std::vector<float> demand(cells);
    cudaMemcpy(demand.data(), view.demand, cells * 4, cudaMemcpyDeviceToHost);
    cudb::RoutingStatistics stats;
    cudaMemcpy(&stats, view.statistics, sizeof(stats), cudaMemcpyDeviceToHost);
    state.download_routes(false);
    dump(dir, "z_routes", state.routes_cpu.get(), view.ROUTE_PER_PIN * view.PIN_NUM + 1);
    dump(dir, "z_demand", demand);
    std::vector<double> st{stats.total_wirelength, double(stats.total_via_count), double(state.global_timestamp),
                           double(status)};
    dump(dir, "z_stats", st);
    printf("REF_ZSHAPE nets=%zu groups=%zu batches=%zu status=%d\n", order.size(), groups.size(), batches.size(), status);
    memory.clear();
    state.release_workspaces();
    return 0;
}
#endif

int run_batch(const std::string& dir, int limit, int sparsity) {
    const auto meta = load<int>(dir + "/meta.i32");
    const auto order = load<int>(dir + "/order.i32");
    const auto point_off = load<int>(dir + "/point_off.i32"), points = load<int>(dir + "/points.i32");
    const auto hseg_off = load<int>(dir + "/hseg_off.i32"), hsegs = load<int>(dir + "/hsegs.i32");
    const auto vseg_off = load<int>(dir + "/vseg_off.i32"), vsegs = load<int>(dir + "/vsegs.i32");
    cudb::RouterState state;
    state.device.X = meta[1];
    state.device.Y = meta[2];
    const int n = point_off.size() - 1;
    state.nets.resize(n);
    for (int i = 0; i < n; ++i) {
        auto& net = state.nets[i];
        net.points.assign(points.begin() + point_off[i], points.begin() + point_off[i + 1]);
        for (int s = hseg_off[i]; s < hseg_off[i + 1]; ++s) net.rsmt_h_segments.emplace_back(hsegs[2 * s], hsegs[2 * s + 1]);
        for (int s = vseg_off[i]; s < vseg_off[i + 1]; ++s) net.rsmt_v_segments.emplace_back(vsegs[2 * s], vsegs[2 * s + 1]);
    }
    std::vector<int> sorted = order;
    const auto start = std::chrono::steady_clock::now();
    auto batches = cudb::generate_batches_rsmt(state, sorted, limit, sparsity);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    std::vector<int> batch_of(order.size(), -1), pos(n, -1);
    for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = i;
    for (size_t b = 0; b < batches.size(); ++b)
        for (int id : batches[b]) batch_of[pos[id]] = int(b);
    dump(dir, "ref_batch_of", batch_of);
    printf("REF_BATCH nets=%zu batches=%zu elapsed_ms=%.6f\n", order.size(), batches.size(), ms);
    return 0;
}

int run_write(const std::string& cap, const std::string& net, const std::string& dir, const std::string& lut,
              const std::string& routes_path, const std::string& out) {
    read_design(cap, net, lut);
    cudb::RouterState state;
    cudb::prepare_routing_nets(state);
    const auto words = load<int>(routes_path);
    state.routes_cpu.reset(new int[words.size()]);
    std::copy(words.begin(), words.end(), state.routes_cpu.get());
    for (int i = 0; i < int(db::nets.size()); ++i)
        if (db::nets[i].pins.size() == 1) nets2output.push(i);
    // Lshape_route leaves nets2route in plan order and finish_nets publishes in
    // that order (lshape.cuh:70-77, pipeline.hpp:77): use the plan if given.
    std::vector<int> all(state.nets.size());
    std::iota(all.begin(), all.end(), 0);
    if (std::filesystem::exists(dir + "/ids.i32")) all = load<int>(dir + "/ids.i32");
    out_file = fopen(out.c_str(), "w");
    if (!out_file) throw std::runtime_error("cannot open " + out);
    setvbuf(out_file, nullptr, _IONBF, 0);
    graph::finish_nets(state, all);
    auto records = graph::collect_output_nets(std::move(nets2output));
    nets2output = {};
    graph::output_nets(state, std::move(records));
    fclose(out_file);
    out_file = nullptr;
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        program_start = std::chrono::high_resolution_clock::now();
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "topo" && argc == 6) return run_topo(argv[2], argv[3], argv[4], argv[5]);
        if (mode == "route" && argc == 7) return run_route(argv[2], argv[3], argv[4], argv[5], argv[6]);
        if (mode == "snap" && argc == 7) return run_snap(argv[2], argv[3], argv[4], argv[5], std::stoi(argv[6]));
        if (mode == "flt" && argc == 6) return run_flt(argv[2], argv[3], argv[4], argv[5]);
#ifdef GROTOR_GGR_ROUTING
        if (mode == "zshape" && argc == 6) return run_zshape(argv[2], argv[3], argv[4], argv[5]);
#endif
        if (mode == "batch" && argc == 5) return run_batch(argv[2], std::stoi(argv[3]), std::stoi(argv[4]));
        if (mode == "write" && argc == 8) return run_write(argv[2], argv[3], argv[4], argv[5], argv[6], argv[7]);
        fprintf(stderr, "usage: ref_harness topo|route|snap|flt|zshape|batch|write ...\n");
        return 2;
    } catch (const std::exception& e) {
        fprintf(stderr, "ref_harness error: %s\n", e.what());
        return 1;
    }
}
