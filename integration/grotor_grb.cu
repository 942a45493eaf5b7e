// grotor_grb.cu -- the reference router's default pipeline with its routing
// hot path on grotor_b200.
//
// This is the reference-side driver a maintainer of the reference router adds
// to adopt grotor_b200: the program below is the reference's own `main`
// (src/main.cu:22-179) and `grotor::route` (src/pipeline.hpp:14-157), compiled
// against the reference's headers (include path only; nothing is copied), with
// the hot path of its two routing stages replaced by calls into libgrb (the C
// ABI of include/grb.h):
//
//   * stage one, Lshape_route (src/routing/lshape.cuh:21-197): the reference's
//     host code builds the FLUTE trees and the HPWL order as before; the
//     trees' batching geometry and depth-first flattening (construct_rsmt's
//     geometry, lshape.cuh:85-98) are built on the device by
//     grb_build_topology; first-fit batching (generate_batches_cpu_timed),
//     the per-batch cost refresh, the L-shape DP and the demand commit run in
//     grb_plan_batches + grb_lshape_stage, whose stage tail also computes the
//     congestion view and the rip-up classification the pipeline needs next
//     (pipeline.hpp:86-93);
//   * stage two, Lshape_route_detour::route_detour (src/routing/flt.cuh:
//     186-192): the reference's host FLT DAG builder (process_net,
//     flt.cuh:8-46) runs unchanged on the congestion view; batching and the
//     DAG execution loop of route_prepared_topology (flt.cuh:75-182) run in
//     grb_plan_batches + grb_upload_flt + grb_flt_stage;
//   * the .out writer, graph::output_nets (src/output.hpp:79-112): the text of
//     each part of the file is formatted on the device from the device's
//     routes (grb_format_out) and drained into the file by a host task
//     (grb_drain_out) that overlaps the next stage, where the reference's
//     output task (pipeline.hpp:20-35) formats on the host.
//
// Everything else -- CAP/NET parsing (db::read), net splitting
// (prepare_routing_nets), FLUTE, the FLT DAG builder, finish_nets and
// collect_output_nets -- is the reference's code, so the same input gives the
// same .out (stage-one nets byte for byte; for stage-two nets the reference's
// own segment order is not defined, so the segments of each net are compared
// as a set).
//
// Usage: grotor_grb -cap FILE -net FILE -out FILE [--lut-dir DIR]
//                   [--executor persistent|plain|graph] [--stop-after lshape|routing]
//                   [--report-traffic 0|1]
#include "pipeline.hpp"

#include <filesystem>
#include <future>

#include "drop_in.cuh"
#include "grb_prof.h"

namespace drop_in {

// --report-traffic 1: print the FLT stage's algorithmic bytes (grb_flt_traffic)
// beside its timing, for its roofline.
bool report_traffic = false;

// Stage one: Lshape_route (lshape.cuh:21-197) with batching, cost refresh,
// DAG and commit on grotor_b200.  Leaves nets2route in the plan order, as
// the reference does.
void lshape_stage(cudb::RouterState& state, grb_ctx* ctx, std::vector<int>& nets2route, int32_t mode,
                  int64_t initial_vias, bool tail) {
    auto& nets = state.nets;
    const auto topology_start = std::chrono::steady_clock::now();
    // FLUTE only (construct_rsmt's rsmt_only form); the geometry and the
    // depth-first trees are built on the device.
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < int(nets2route.size()); ++i) nets[nets2route[i]].construct_rsmt(state, true);
    Trees F = flatten_trees(state);
    check(grb_build_topology(ctx, &F.t), ctx, "grb_build_topology");
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
    std::vector<int32_t> batch_off(nb + 1);
    int32_t n = 0, nb2 = 0;
    check(grb_get_plan(ctx, nets2route.data(), batch_off.data(), &n, &nb2), ctx, "grb_get_plan");
    if (report_traffic) {  // the .out is written from the device's routes; the host copy feeds the byte model
        const size_t words = size_t(state.device.ROUTE_PER_PIN) * state.device.PIN_NUM + 1;
        state.routes_cpu.reset(new int[words]());
        check(grb_read_routes(ctx, state.routes_cpu.get()), ctx, "grb_read_routes");
    }
    printf("DAG_TIMING stage=lshape batch_index=-1 elapsed_ms=%.6f nets=%zu batches=%d executor=grotor_b200\n",
           st.dag_ms, nets2route.size(), nb);
    printf("BATCH_TIMING backend=grotor_b200 elapsed_ms=%.6f nets=%zu batches=%d used_for_routing=1\n",
           st.batching_ms, nets2route.size(), nb);
}

// Stage two: Lshape_route_detour::route_detour (flt.cuh:186-192).  The
// congestion view comes from the stage tail; the host DAG builder is the
// reference's; batching and route_prepared_topology's batch loop run on
// grotor_b200.
void flt_stage(cudb::RouterState& state, grb_ctx* ctx, const grb_grid& grid, std::vector<int>& nets2route, int32_t mode,
               std::vector<unsigned char>& cong, std::vector<float>& xsum, std::vector<float>& ysum) {
    if (nets2route.empty()) return;
    auto& nets = state.nets;
    // prepare_detour_topology (flt.cuh:48-73) with the view in host memory.
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
    // The FLT DAGs (flt::Topology spans) and batching geometry, by net id.
    const int count = int(nets.size());
    std::vector<int> slot_of(count, -1);
    for (size_t s = 0; s < nets2route.size(); ++s) slot_of[nets2route[s]] = int(s);
    std::vector<int32_t> node_off{0}, coord, depth, children, parent_end, edge_off{0}, edge_parent, edge_slot;
    std::vector<int32_t> point_off{0}, points, hseg_off{0}, hsegs, vseg_off{0}, vsegs;
    std::vector<int64_t> route2_off{0};
    const auto& topo = state.flt_topology;
    for (int id = 0; id < count; ++id) {
        const int s = slot_of[id];
        if (s >= 0) {
            const auto& span = topo.spans[s];
            const auto& arena = topo.arenas[span.lane];
            for (int i = 0; i < span.nodes; ++i) {
                const auto& nd = arena.nodes[span.node_begin + i];
                coord.push_back(nd.coordinate);
                depth.push_back(nd.depth);
                children.push_back(nd.children);
                parent_end.push_back(nd.parent_end);
            }
            for (int i = 0; i < span.edges; ++i) {
                const auto& e = arena.edges[span.edge_begin + i];
                edge_parent.push_back(e.parent);
                edge_slot.push_back(e.source_slot);
            }
        }
        node_off.push_back(int32_t(coord.size()));
        edge_off.push_back(int32_t(edge_parent.size()));
        const auto& n = nets[id];
        for (int p : n.points) points.push_back(p);
        point_off.push_back(int32_t(points.size()));
        for (const auto& sg : n.rsmt_h_segments) { hsegs.push_back(sg.first); hsegs.push_back(sg.second); }
        hseg_off.push_back(int32_t(hsegs.size() / 2));
        for (const auto& sg : n.rsmt_v_segments) { vsegs.push_back(sg.first); vsegs.push_back(sg.second); }
        vseg_off.push_back(int32_t(vsegs.size() / 2));
        const int64_t words = s >= 0 ? int64_t(n.pins.size()) * int64_t(state.device.ROUTE_PER_PIN_PHASE2) : 0;
        route2_off.push_back(route2_off.back() + words);
    }
    state.flt_topology.clear();
    check(grb_upload_geometry(ctx, point_off.data(), points.data(), hseg_off.data(), hsegs.data(), vseg_off.data(),
                              vsegs.data()),
          ctx, "grb_upload_geometry");
    int32_t nb = 0;
    check(grb_plan_batches(ctx, nets2route.data(), int32_t(nets2route.size()), 300000, state.batch_sparsity_override,
                           mode == GRB_MODE_PERSISTENT ? GRB_MODE_PERSISTENT : GRB_MODE_PLAIN, nullptr, &nb),
          ctx, "grb_plan_batches (FLT)");
    grb_flt_dags d{node_off.data(), coord.data(), depth.data(), children.data(), parent_end.data(),
                   edge_off.data(), edge_parent.data(), edge_slot.data(), route2_off.data()};
    check(grb_upload_flt(ctx, &d), ctx, "grb_upload_flt");
    grb_stats st{};
    check(grb_flt_stage(ctx, 1, mode, &st), ctx, "grb_flt_stage");
    if (report_traffic) {
        const size_t words = size_t(state.device.ROUTE_PER_PIN_PHASE2) * state.device.PIN_NUM_PHASE2 + 1;
        state.routes_phase2_cpu.reset(new int[std::max<size_t>(words, size_t(route2_off.back()) + 1)]());
        check(grb_read_routes2(ctx, state.routes_phase2_cpu.get()), ctx, "grb_read_routes2");
    }
    printf("DAG_TIMING stage=detour batch_index=-1 elapsed_ms=%.6f nets=%zu batches=%d executor=grotor_b200\n",
           st.dag_ms, nets2route.size(), nb);
    printf("BATCH_TIMING stage=detour backend=grotor_b200 elapsed_ms=%.6f nets=%zu batches=%d used_for_routing=1\n",
           st.batching_ms, nets2route.size(), nb);
    if (report_traffic) {
        std::vector<int32_t> plan(nets2route.size()), plan_off(size_t(nb) + 1);
        int32_t pn = 0, pb = 0;
        check(grb_get_plan(ctx, plan.data(), plan_off.data(), &pn, &pb), ctx, "grb_get_plan");
        std::vector<int64_t> route_off(size_t(count) + 1);
        for (int id = 0; id <= count; ++id)
            route_off[id] = int64_t(state.pin_cnt_sum_cpu[id]) * int64_t(state.device.ROUTE_PER_PIN);
        double bytes[3] = {0, 0, 0};
        check(grb_flt_traffic(&grid, pb, plan_off.data(), plan.data(), &d, route_off.data(), state.routes_cpu.get(),
                              state.routes_phase2_cpu.get(), 1, bytes), ctx, "grb_flt_traffic");
        printf("FLT_TRAFFIC refresh_bytes=%.0f dp_bytes=%.0f commit_bytes=%.0f\n", bytes[0], bytes[1], bytes[2]);
    }
}

// grotor::route (pipeline.hpp:14-157).  The output order is the reference's:
// single-pin nets, then (after stage one) the nets without overflow, then the
// rerouted ones.
void route(cudb::RouterState& state, int32_t mode, bool stop_after_lshape) {
    cudb::prepare_routing_nets(state);
    int64_t initial_vias = 0;  // one via per metal1 pin (preprocess.hpp:1716-1718)
    for (auto& dbnet : db::nets)
        for (int pin : dbnet.pins) initial_vias += pin < state.device.X * state.device.Y;
    Grid G = make_grid(state);
    grb_ctx* ctx = nullptr;
    check(grb_create(&G.g, 0, &ctx), nullptr, "grb_create");
    std::unique_ptr<grb_ctx, void (*)(grb_ctx*)> owner(ctx, grb_destroy);
    Output out{ctx};
    // Single-pin nets first (pipeline.hpp:57-59), written while stage one runs.
    for (int i = 0; i < int(db::nets.size()); ++i)
        if (db::nets[i].pins.size() == 1) nets2output.push(i);
    out.start(state);
    std::vector<int> all_nets(state.nets.size());
    std::iota(all_nets.begin(), all_nets.end(), 0);
    lshape_stage(state, ctx, all_nets, mode, initial_vias, !stop_after_lshape);
    if (stop_after_lshape) {
        graph::finish_nets(state, all_nets);
        out.start(state);
        out.wait();
        return;
    }
    // pipeline.hpp:86-106: classification, phase-two offsets (the global
    // `mode` of runtime.hpp:29 selects the DAG builder's variant for large
    // designs).
    if (state.nets.size() > 5000000) ::mode = 1;
    if (state.nets.size() > 20000000) ::mode = 2;
    const size_t xy = size_t(state.device.X) * state.device.Y;
    std::vector<unsigned char> is_of(state.nets.size()), cong(xy);
    std::vector<float> xsum(xy), ysum(xy);
    check(grb_read_stage_tail(ctx, is_of.data(), cong.data(), xsum.data(), ysum.data()), ctx, "grb_read_stage_tail");
    std::vector<int> of_nets, no_of_nets;
    for (int i = 0; i < int(is_of.size()); ++i) (is_of[i] ? of_nets : no_of_nets).push_back(i);
    graph::finish_nets(state, no_of_nets);
    int pin_count = 0;
    for (int id : of_nets) {
        state.pin_cnt_sum_phase2_cpu[id] = pin_count;
        pin_count += int(state.nets[id].pins.size());
        state.ripup_flag_cpu[id] = 1;
    }
    state.device.PIN_NUM_PHASE2 = pin_count;
    // The nets without overflow are written while stage two runs, as the
    // reference's output task does (pipeline.hpp:108-109).
    out.start(state);
    // Stage two sorts of_nets in place (flt.cuh:52), and the reference
    // publishes the rerouted nets in that order (pipeline.hpp:137,143).
    flt_stage(state, ctx, G.g, of_nets, mode, cong, xsum, ysum);
    graph::finish_nets(state, of_nets);
    out.start(state);
    out.wait();
    printf("OUTPUT_TIMING format_ms=%.3f output_wait_ms=%.3f executor=grotor_b200\n", out.format_ms, out.wait_ms);
}

}  // namespace drop_in

int main(int argc, char** argv) {
    try {
        std::string cap, net, output, lut_dir = ".", executor = "persistent";
        bool stop_after_lshape = false;
        if (argc < 7 || argc % 2 != 1)
            throw std::invalid_argument("Usage: grotor_grb -cap FILE -net FILE -out FILE [--lut-dir DIR] "
                                        "[--executor persistent|plain|graph] [--stop-after lshape|routing] "
                                        "[--report-traffic 0|1]");
        for (int i = 1; i < argc; i += 2) {
            const std::string option = argv[i], value = argv[i + 1];
            if (option == "-cap") cap = value;
            else if (option == "-net") net = value;
            else if (option == "-out") output = value;
            else if (option == "--lut-dir") lut_dir = value;
            else if (option == "--executor") executor = value;
            else if (option == "--report-traffic") drop_in::report_traffic = value == "1";
            else if (option == "--stop-after") {
                if (value != "lshape" && value != "routing") throw std::invalid_argument("--stop-after expects lshape or routing");
                stop_after_lshape = value == "lshape";
            } else throw std::invalid_argument("Unknown option: " + option);
        }
        if (cap.empty() || net.empty() || output.empty()) throw std::invalid_argument("-cap, -net and -out are required");
        const int32_t mode = drop_in::executor_mode(executor);
        program_start = std::chrono::high_resolution_clock::now();
        db::read(cap.data(), net.data());
        const auto caller_directory = std::filesystem::current_path();
        std::filesystem::current_path(lut_dir);
        flute::readLUT();
        std::filesystem::current_path(caller_directory);
        out_file = fopen(output.c_str(), "w");
        if (!out_file) throw std::runtime_error("Cannot open output: " + output);
        if (setvbuf(out_file, nullptr, _IONBF, 0)) throw std::runtime_error("Cannot configure routing output");
        {
            cudb::RouterState state;
            state.batch_sparsity_override = 1;
            state.report_score = false;
            drop_in::route(state, mode, stop_after_lshape);
        }
        const int close_status = fclose(out_file);
        out_file = nullptr;
        if (close_status) throw std::runtime_error("Failed to close routing output");
        printf("GROTOR_COMPLETE wall_seconds=%.6f\n", elapsed_time());
        return EXIT_SUCCESS;
    } catch (const std::exception& error) {
        if (out_file) fclose(out_file);
        fprintf(stderr, "grotor_grb error: %s\n", error.what());
        return EXIT_FAILURE;
    }
}
