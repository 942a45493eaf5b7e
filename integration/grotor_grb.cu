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
//                   [--flt-block-width N]
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

// Stage two: Lshape_route_detour::route_detour (flt.cuh:186-192).  The
// congestion view comes from the stage tail; the host DAG builder is the
// reference's; batching and route_prepared_topology's batch loop run on
// grotor_b200.
void flt_stage(cudb::RouterState& state, grb_ctx* ctx, const grb_grid& grid, std::vector<int>& nets2route, int32_t mode,
               std::vector<unsigned char>& cong, std::vector<float>& xsum, std::vector<float>& ysum) {
    if (nets2route.empty()) return;
    detour_prepare(state, nets2route, cong, xsum, ysum);
    phases.mark("flt_prepare");
    FltRun run = flt_run(state, ctx, nets2route, mode, 1, state.device.ROUTE_PER_PIN_PHASE2, "detour");
    if (report_traffic) {
        const int count = int(state.nets.size());
        const size_t words = size_t(state.device.ROUTE_PER_PIN_PHASE2) * state.device.PIN_NUM_PHASE2 + 1;
        state.routes_phase2_cpu.reset(new int[std::max<size_t>(words, size_t(run.route2_off.back()) + 1)]());
        check(grb_read_routes2(ctx, state.routes_phase2_cpu.get()), ctx, "grb_read_routes2");
        const int32_t nb = run.nb;
        const grb_flt_dags& d = run.d;
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
    Phases& ph = phases;
    cudb::prepare_routing_nets(state);
    ph.mark("prepare");
    int64_t initial_vias = 0;  // one via per metal1 pin (preprocess.hpp:1716-1718)
    for (auto& dbnet : db::nets)
        for (int pin : dbnet.pins) initial_vias += pin < state.device.X * state.device.Y;
    Grid G = make_grid(state);
    grb_ctx* ctx = nullptr;
    check(grb_create(&G.g, 0, &ctx), nullptr, "grb_create");
    std::unique_ptr<grb_ctx, void (*)(grb_ctx*)> owner(ctx, grb_destroy);
    ph.mark("create");
    Output out{ctx};
    // Single-pin nets first (pipeline.hpp:57-59), written while stage one runs.
    for (int i = 0; i < int(db::nets.size()); ++i)
        if (db::nets[i].pins.size() == 1) nets2output.push(i);
    out.start(state);
    ph.mark("output_first");
    std::vector<int> all_nets(state.nets.size());
    std::iota(all_nets.begin(), all_nets.end(), 0);
    lshape_stage(state, ctx, all_nets, mode, initial_vias, !stop_after_lshape, report_traffic);
    ph.mark("lshape_rest");
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
    ph.mark("classification");
    // The nets without overflow are written while stage two runs, as the
    // reference's output task does (pipeline.hpp:108-109).
    out.start(state);
    ph.mark("output_start");
    // Stage two sorts of_nets in place (flt.cuh:52), and the reference
    // publishes the rerouted nets in that order (pipeline.hpp:137,143).
    flt_stage(state, ctx, G.g, of_nets, mode, cong, xsum, ysum);
    ph.mark("flt_rest");
    graph::finish_nets(state, of_nets);
    out.start(state);
    out.wait();
    ph.mark("output_finish");
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
                                        "[--flt-block-width N] "
                                        "[--report-traffic 0|1]");
        for (int i = 1; i < argc; i += 2) {
            const std::string option = argv[i], value = argv[i + 1];
            if (option == "-cap") cap = value;
            else if (option == "-net") net = value;
            else if (option == "-out") output = value;
            else if (option == "--lut-dir") lut_dir = value;
            else if (option == "--executor") executor = value;
            else if (option == "--report-traffic") drop_in::report_traffic = value == "1";
            else if (option == "--flt-block-width") drop_in::flt_block_width = std::stoi(value);
            else if (option == "--stop-after") {
                if (value != "lshape" && value != "routing") throw std::invalid_argument("--stop-after expects lshape or routing");
                stop_after_lshape = value == "lshape";
            } else throw std::invalid_argument("Unknown option: " + option);
        }
        if (cap.empty() || net.empty() || output.empty()) throw std::invalid_argument("-cap, -net and -out are required");
        const int32_t mode = drop_in::executor_mode(executor);
        program_start = std::chrono::high_resolution_clock::now();
        drop_in::Phases& ph = drop_in::phases;
        ph.last = program_start;
        // CUDA starts while the input is read (src/main.cu:101-106).
        auto gpu_ready = std::async(std::launch::async, [] { return grb_init_device(0); });
        db::read(cap.data(), net.data());
        ph.mark("read");
        const auto caller_directory = std::filesystem::current_path();
        std::filesystem::current_path(lut_dir);
        flute::readLUT();
        std::filesystem::current_path(caller_directory);
        out_file = fopen(output.c_str(), "w");
        if (!out_file) throw std::runtime_error("Cannot open output: " + output);
        if (setvbuf(out_file, nullptr, _IONBF, 0)) throw std::runtime_error("Cannot configure routing output");
        ph.mark("lut");
        drop_in::check(gpu_ready.get(), nullptr, "grb_init_device");
        ph.mark("cuda_init_wait");
        {
            cudb::RouterState state;
            state.batch_sparsity_override = 1;
            state.report_score = false;
            drop_in::route(state, mode, stop_after_lshape);
        }
        ph.mark("teardown");
        const int close_status = fclose(out_file);
        out_file = nullptr;
        if (close_status) throw std::runtime_error("Failed to close routing output");
        ph.print();
        printf("GROTOR_COMPLETE wall_seconds=%.6f\n", elapsed_time());
        return EXIT_SUCCESS;
    } catch (const std::exception& error) {
        if (out_file) fclose(out_file);
        fprintf(stderr, "grotor_grb error: %s\n", error.what());
        return EXIT_FAILURE;
    }
}
