// grotor_grb_cugr2.cu -- the reference router's CUGR2 pipeline with its
// routing hot path on grotor_b200.
//
// The reference's own `main` (src/main.cu:22-179) and `grotor::route_cugr2`
// (src/pipeline_cugr2.hpp:65-131), compiled against the reference's headers
// with GROTOR_CUGR2_ROUTING (the defines of its grotor_cugr2 build; include
// path only, nothing is copied):
//
//   * stage one (L-shape) and its congestion view and rip-up set run as in
//     the default drop-in (integration/drop_in.cuh);
//   * stage two, route_detour on the rip-up set, with phase-two storage of at
//     least 128 words per pin (reserve_reroute_storage,
//     pipeline_cugr2.hpp:14-63): the reference's FLT DAG builder, then
//     batching and the FLT batch loop on grotor_b200;
//   * the maze stage on the nets still overflowing (pipeline_cugr2.hpp:90-117):
//     the checkpoint and score gate (grb_checkpoint, grb_routing_score,
//     grb_restore), the reference's host sparse-maze topology
//     (maze::prepare_topology), the removal of the nets' routes
//     (grb_remove_routes, maze::remove_routes) and the FLT executor on the maze
//     DAGs without stage-one rip-up (grb_flt_stage, remove_phase_one = 0);
//   * the output: the reference's writer on the downloaded routes, as its
//     CUGR2 pipeline does.
//
// Usage: grotor_grb_cugr2 -cap FILE -net FILE -out FILE [--lut-dir DIR]
//                         [--executor persistent|plain|graph]
#include "pipeline_cugr2.hpp"

#include <cmath>
#include <filesystem>

#include "drop_in.cuh"

namespace drop_in {

// reserve_reroute_storage (pipeline_cugr2.hpp:14-63) on the host copy of the
// phase-two routes: nets not yet flagged get offsets after the current ones;
// the stride grows to `minimum` and the flagged nets' words move to the new
// layout.
void reserve_phase2(cudb::RouterState& state, const std::vector<int>& ids, int64_t minimum) {
    auto& view = state.device;
    const int old_pins = view.PIN_NUM_PHASE2;
    const int64_t old_stride = view.ROUTE_PER_PIN_PHASE2;
    for (int id : ids)
        if (!state.ripup_flag_cpu[id]) {
            state.pin_cnt_sum_phase2_cpu[id] = view.PIN_NUM_PHASE2;
            view.PIN_NUM_PHASE2 += int(state.nets[id].pins.size());
            state.ripup_flag_cpu[id] = 1;
        }
    const int64_t stride = std::max<int64_t>(old_stride, minimum);
    std::unique_ptr<int[]> fresh(new int[size_t(stride) * view.PIN_NUM_PHASE2 + 1]());
    if (old_pins && state.routes_phase2_cpu)
        for (int id = 0; id < int(state.nets.size()); ++id) {
            const int offset = state.pin_cnt_sum_phase2_cpu[id];
            if (!state.ripup_flag_cpu[id] || offset >= old_pins) continue;
            std::copy_n(state.routes_phase2_cpu.get() + size_t(offset) * old_stride,
                        state.nets[id].pins.size() * size_t(old_stride), fresh.get() + size_t(offset) * stride);
        }
    state.routes_phase2_cpu = std::move(fresh);
    view.ROUTE_PER_PIN_PHASE2 = int(stride);
    printf("REROUTE_STORAGE pins=%d stride=%lld bytes=%llu\n", view.PIN_NUM_PHASE2, (long long)stride,
           (unsigned long long)((stride * view.PIN_NUM_PHASE2 + 1) * sizeof(int)));
}

// Host phase-two routes (laid out at offsets * stride, for the nets in
// `flags`) into the device store laid out by run.route2_off.
void store_phase2(grb_ctx* ctx, const cudb::RouterState& state, const FltRun& run, const int* routes, int64_t stride,
                  const std::vector<int>& offsets, const std::vector<int>& flags) {
    std::vector<int32_t> words(size_t(run.route2_off.back()) + 1, 0);
    for (int id = 0; id < int(state.nets.size()); ++id) {
        const int64_t slot = run.route2_off[id + 1] - run.route2_off[id];
        if (!flags[id] || !slot) continue;
        const int64_t n = std::min<int64_t>(slot, int64_t(state.nets[id].pins.size()) * stride);
        std::copy_n(routes + size_t(offsets[id]) * stride, n, words.data() + run.route2_off[id]);
    }
    check(grb_write_routes2(ctx, words.data()), ctx, "grb_write_routes2");
}

// The phase-two words of the stage just run (laid out by run.route2_off) into
// the host copy at the reference's offsets.
void collect_phase2(cudb::RouterState& state, grb_ctx* ctx, const FltRun& run, const std::vector<int>& ids) {
    std::vector<int32_t> words(size_t(run.route2_off.back()) + 1);
    check(grb_read_routes2(ctx, words.data()), ctx, "grb_read_routes2");
    const int64_t stride = state.device.ROUTE_PER_PIN_PHASE2;
    for (int id : ids) {
        const int64_t n = run.route2_off[id + 1] - run.route2_off[id];
        std::copy_n(words.data() + run.route2_off[id], n,
                    state.routes_phase2_cpu.get() + size_t(state.pin_cnt_sum_phase2_cpu[id]) * stride);
    }
}

// Device tables that maze::MazeCostView reads through the reference's
// device view (capacity, demand, edge lengths, overflow weights) and the
// unit costs it reads from the view itself.
struct MazeView {
    float *capacity = nullptr, *demand = nullptr;
    int *xlen = nullptr, *ylen = nullptr;
    double* short_costs = nullptr;
    ~MazeView() {
        for (void* p : {(void*)capacity, (void*)demand, (void*)xlen, (void*)ylen, (void*)short_costs})
            if (p) cudaFree(p);
    }
};

void maze_view(cudb::RouterState& state, grb_ctx* ctx, const Grid& G, MazeView& M) {
    const size_t cells = G.capacity.size();
    auto up = [&](auto*& dst, const auto& src) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(dst)>>;
        if (!dst) grotor::cuda_check(cudaMalloc(&dst, std::max<size_t>(src.size(), 1) * sizeof(T)), "maze view");
        grotor::cuda_check(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice), "maze view");
    };
    std::vector<int32_t> half(cells);
    check(grb_read_tables(ctx, nullptr, nullptr, nullptr, half.data(), nullptr), ctx, "grb_read_tables");
    std::vector<float> demand(cells);
    for (size_t i = 0; i < cells; ++i) demand[i] = float(half[i]) * 0.5f;
    up(M.capacity, G.capacity);
    up(M.demand, demand);
    up(M.xlen, G.xlen);
    up(M.ylen, G.ylen);
    up(M.short_costs, G.short_costs);
    auto& view = state.device;
    view.unit_length_wire_cost = db::unit_length_wire_cost;  // build_cuda_database, preprocess.hpp:1678-1679
    view.unit_via_cost = db::unit_via_cost;
    view.capacity = M.capacity;
    view.demand = M.demand;
    view.x_edge_len = M.xlen;
    view.y_edge_len = M.ylen;
    view.unit_length_short_costs = M.short_costs;
}

void route_cugr2(cudb::RouterState& state, int32_t mode) {
    cudb::prepare_routing_nets(state);
    phases.mark("prepare");
    int64_t initial_vias = 0;  // one via per metal1 pin (preprocess.hpp:1716-1718)
    for (auto& dbnet : db::nets)
        for (int pin : dbnet.pins) initial_vias += pin < state.device.X * state.device.Y;
    Grid G = make_grid(state);
    grb_ctx* ctx = nullptr;
    check(grb_create(&G.g, 0, &ctx), nullptr, "grb_create");
    std::unique_ptr<grb_ctx, void (*)(grb_ctx*)> owner(ctx, grb_destroy);
    phases.mark("create");
    for (int i = 0; i < int(db::nets.size()); ++i)
        if (db::nets[i].pins.size() == 1) nets2output.push(i);
    const int count = int(state.nets.size());
    std::vector<int> all_nets(count);
    std::iota(all_nets.begin(), all_nets.end(), 0);
    printf("ROUTING_STAGE_BEGIN stage=lshape nets=%zu\n", all_nets.size());
    lshape_stage(state, ctx, all_nets, mode, initial_vias, true, true);
    printf("ROUTING_STAGE_END stage=lshape\n");
    phases.mark("lshape_rest");
    if (state.nets.size() > 5000000) ::mode = 1;
    if (state.nets.size() > 20000000) ::mode = 2;
    const size_t xy = size_t(state.device.X) * state.device.Y;
    std::vector<unsigned char> is_of(count), cong(xy);
    std::vector<float> xsum(xy), ysum(xy);
    check(grb_read_stage_tail(ctx, is_of.data(), cong.data(), xsum.data(), ysum.data()), ctx, "grb_read_stage_tail");
    std::vector<int> detour;
    for (int i = 0; i < count; ++i) if (is_of[i]) detour.push_back(i);
    reserve_phase2(state, detour, 128);
    phases.mark("classification");
    printf("ROUTING_STAGE_BEGIN stage=detour nets=%zu\n", detour.size());
    if (!detour.empty()) {
        detour_prepare(state, detour, cong, xsum, ysum);
        phases.mark("flt_prepare");
        FltRun run = flt_run(state, ctx, detour, mode, 1, state.device.ROUTE_PER_PIN_PHASE2, "detour");
        collect_phase2(state, ctx, run, detour);
    }
    phases.mark("detour_collect");
    printf("ROUTING_STAGE_END stage=detour\n");

    // pipeline_cugr2.hpp:90-117: the maze stage on the nets still overflowing
    // (classified on each net's current route).
    std::vector<uint8_t> flag(count);
    for (int i = 0; i < count; ++i) flag[i] = state.ripup_flag_cpu[i] != 0;
    check(grb_ripup_classify_phase2(ctx, 0, flag.data(), is_of.data()), ctx, "grb_ripup_classify_phase2");
    std::vector<int> maze_nets;
    for (int i = 0; i < count; ++i) if (is_of[i]) maze_nets.push_back(i);
    printf("ROUTING_STAGE_BEGIN stage=maze nets=%zu\n", maze_nets.size());
    const auto maze_start = std::chrono::steady_clock::now();
    if (!maze_nets.empty()) {
        // checkpoint: device demand and statistics, host flags, offsets and routes
        check(grb_checkpoint(ctx), ctx, "grb_checkpoint");
        const auto flags = state.ripup_flag_cpu;
        const auto offsets = state.pin_cnt_sum_phase2_cpu;
        const int pins = state.device.PIN_NUM_PHASE2;
        const int stride0 = state.device.ROUTE_PER_PIN_PHASE2;
        const size_t words0 = size_t(stride0) * pins + 1;
        std::unique_ptr<int[]> routes0(new int[words0]);
        std::copy_n(state.routes_phase2_cpu.get(), words0, routes0.get());
        phases.mark("maze_checkpoint");
        double before = 0;
        check(grb_routing_score(ctx, &before), ctx, "grb_routing_score");
        MazeView M;
        maze_view(state, ctx, G, M);
        phases.mark("maze_view");
        grotor::maze::prepare_topology(state, maze_nets);
        phases.mark("maze_search");
        std::vector<uint8_t> phase2(maze_nets.size());
        for (size_t k = 0; k < maze_nets.size(); ++k) phase2[k] = state.ripup_flag_cpu[maze_nets[k]] != 0;
        check(grb_remove_routes(ctx, maze_nets.data(), int32_t(maze_nets.size()), phase2.data()), ctx,
              "grb_remove_routes");
        int64_t stride = 128;
        for (int id : maze_nets) {
            const int64_t words = 10ll * int64_t(state.nets[id].rsmt.back().size()) + 1;
            const int64_t p = int64_t(state.nets[id].pins.size());
            stride = std::max(stride, (words + p - 1) / p);
        }
        reserve_phase2(state, maze_nets, stride);
        phases.mark("maze_remove_reserve");
        // Every flagged net keeps phase-two storage on the device (the earlier
        // stage's routes are written into it), so the score, the final
        // classification and a restore see each net's current route.
        std::vector<uint8_t> keep(count);
        for (int i = 0; i < count; ++i) keep[i] = state.ripup_flag_cpu[i] != 0;
        const int64_t stride1 = state.device.ROUTE_PER_PIN_PHASE2;
        FltRun run = flt_run(state, ctx, maze_nets, mode, 0, stride1, "maze", &keep, [&](FltRun& R) {
            store_phase2(ctx, state, R, state.routes_phase2_cpu.get(), stride1, state.pin_cnt_sum_phase2_cpu,
                         state.ripup_flag_cpu);
        });
        collect_phase2(state, ctx, run, maze_nets);
        phases.mark("maze_collect");
        double after = 0;
        check(grb_routing_score(ctx, &after), ctx, "grb_routing_score");
        const bool accepted = std::isfinite(after) && after < before;
        if (!accepted) {
            check(grb_restore(ctx), ctx, "grb_restore");
            store_phase2(ctx, state, run, routes0.get(), stride0, offsets, flags);
            state.ripup_flag_cpu = flags;
            state.pin_cnt_sum_phase2_cpu = offsets;
            state.device.PIN_NUM_PHASE2 = pins;
            state.device.ROUTE_PER_PIN_PHASE2 = stride0;
            state.routes_phase2_cpu = std::move(routes0);
        }
        printf("MAZE_QUALITY_GATE accepted=%d before_score=%.12g candidate_score=%.12g\n", int(accepted), before,
               after);
        phases.mark("maze_gate");
        state.device.capacity = nullptr;
        state.device.demand = nullptr;
        state.device.x_edge_len = state.device.y_edge_len = nullptr;
        state.device.unit_length_short_costs = nullptr;
    }
    printf("MAZE_PHASE_TIMING elapsed_ms=%.6f executor=grotor_b200\n",
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - maze_start).count());
    printf("ROUTING_STAGE_END stage=maze\n");
    for (int i = 0; i < count; ++i) flag[i] = state.ripup_flag_cpu[i] != 0;
    check(grb_ripup_classify_phase2(ctx, 0, flag.data(), is_of.data()), ctx, "grb_ripup_classify_phase2");
    size_t remaining = 0;
    for (unsigned char f : is_of) remaining += f != 0;
    printf("ROUTING_REMAINING_OVERFLOW nets=%zu\n", remaining);
    // pipeline_cugr2.hpp:123-128: the reference's writer on the downloaded routes.
    const size_t words = size_t(state.device.ROUTE_PER_PIN) * state.device.PIN_NUM + 1;
    // Only the words in use move (the writer reads a route below its count
    // word), so the storage needs no clearing.
    state.routes_cpu.reset(new int[words]);
    check(grb_read_routes_used(ctx, state.routes_cpu.get()), ctx, "grb_read_routes_used");
    phases.mark("final_download");
    graph::finish_nets(state, all_nets);
    auto records = graph::collect_output_nets(std::move(nets2output));
    graph::output_nets(state, std::move(records));
    phases.mark("output");
}

}  // namespace drop_in

int main(int argc, char** argv) {
    try {
        std::string cap, net, output, lut_dir = ".", executor = "persistent";
        if (argc < 7 || argc % 2 != 1)
            throw std::invalid_argument("Usage: grotor_grb_cugr2 -cap FILE -net FILE -out FILE [--lut-dir DIR] "
                                        "[--executor persistent|plain|graph]");
        for (int i = 1; i < argc; i += 2) {
            const std::string option = argv[i], value = argv[i + 1];
            if (option == "-cap") cap = value;
            else if (option == "-net") net = value;
            else if (option == "-out") output = value;
            else if (option == "--lut-dir") lut_dir = value;
            else if (option == "--executor") executor = value;
            else throw std::invalid_argument("Unknown option: " + option);
        }
        if (cap.empty() || net.empty() || output.empty()) throw std::invalid_argument("-cap, -net and -out are required");
        const int32_t mode = drop_in::executor_mode(executor);
        program_start = std::chrono::high_resolution_clock::now();
        // CUDA starts while the input is read (src/main.cu:101-106).
        auto gpu_ready = std::async(std::launch::async, [] { return grb_init_device(0); });
        drop_in::phases.last = program_start;
        db::read(cap.data(), net.data());
        drop_in::phases.mark("read");
        const auto caller_directory = std::filesystem::current_path();
        std::filesystem::current_path(lut_dir);
        flute::readLUT();
        std::filesystem::current_path(caller_directory);
        out_file = fopen(output.c_str(), "w");
        if (!out_file) throw std::runtime_error("Cannot open output: " + output);
        if (setvbuf(out_file, nullptr, _IONBF, 0)) throw std::runtime_error("Cannot configure routing output");
        drop_in::phases.mark("lut");
        drop_in::check(gpu_ready.get(), nullptr, "grb_init_device");
        drop_in::phases.mark("cuda_init_wait");
        {
            cudb::RouterState state;
            state.batch_sparsity_override = 1;
            state.report_score = false;
            drop_in::route_cugr2(state, mode);
        }
        drop_in::phases.mark("teardown");
        const int close_status = fclose(out_file);
        out_file = nullptr;
        if (close_status) throw std::runtime_error("Failed to close routing output");
        drop_in::phases.print();
        printf("GROTOR_COMPLETE wall_seconds=%.6f\n", elapsed_time());
        return EXIT_SUCCESS;
    } catch (const std::exception& error) {
        if (out_file) fclose(out_file);
        fprintf(stderr, "grotor_grb_cugr2 error: %s\n", error.what());
        return EXIT_FAILURE;
    }
}
