// grotor_grb_ggr.cu -- the reference router's GGR pipeline with its routing
// hot path on grotor_b200.
//
// The reference's own `main` (src/main.cu:22-179) and `grotor::route_ggr`
// (src/pipeline_ggr.hpp:8-160), compiled against the reference's headers
// with GROTOR_GGR_ROUTING (the defines of its grotor_ggr build; include path
// only, nothing is copied), with the Z-shape stage's hot path replaced by
// calls into libgrb (include/grb.h):
//
//   * FLUTE stays on the host (construct_rsmt's rsmt_only form); the
//     batching geometry is built on the device (grb_build_topology);
//   * first-fit groups (generate_batches_rsmt) and their bounding-box
//     refinement (zshape::generate_bbox_batches, reversed) run in
//     grb_plan_batches + grb_plan_bbox_batches;
//   * the batch loop -- refresh_cost, reset_nodes, solve<4>, convert_routes
//     and the thread-per-net commits (pipeline_ggr.hpp:119-134) -- runs in
//     grb_zshape_stage with the GGR build's integer wire costs
//     (grb_set_wire_cost_mode);
//   * the host post-processing (promote_congested_segments,
//     canonicalize_routes, zshape_topology.hpp:122-248) is the reference's
//     code on the downloaded routes, canonicalize_routes on 8 threads over
//     ranges of nets (only the routes' words in use move, each way:
//     grb_read_routes_used, grb_write_routes_used); the .out is then
//     formatted on the device from the post-processed routes (grb_format_out
//     / grb_drain_out).
//
// Usage: grotor_grb_ggr -cap FILE -net FILE -out FILE [--lut-dir DIR]
//                       [--executor persistent|plain|graph]
#include "pipeline_ggr.hpp"

#include <filesystem>

#include "drop_in.cuh"

namespace drop_in {

// The Z-shape trees in zshape::encode_batch's node order (preorder from the
// tree's first leaf; zshape_topology.hpp:59-121), with each node's 3-D
// position (the encoding itself keeps the 2-D position and the pin layers).
struct ZTrees {
    std::vector<int32_t> node_off{0}, coord, child;
    grb_zshape_trees t{};
};

ZTrees encode_trees(const cudb::RouterState& state) {
    ZTrees Z;
    const auto& view = state.device;
    const int count = int(state.nets.size());
    const std::vector<int> zero(count, 0);
    // Nets in contiguous parts, one per thread, each encoded into its own
    // arrays; the parts are then joined in net order.
    constexpr int kParts = 8;
    struct Part { std::vector<int32_t> size, coord, child; };
    std::vector<Part> parts(kParts);
#pragma omp parallel for num_threads(kParts) schedule(static, 1)
    for (int t = 0; t < kParts; ++t) {
        Part& P = parts[t];
        const int lo = int(int64_t(count) * t / kParts), hi = int(int64_t(count) * (t + 1) / kParts);
        std::vector<int> ord, parent, stack;
        for (int id = lo; id < hi; ++id) {
            const auto& nt = state.nets[id];
            const auto enc = grotor::zshape::encode_batch({id}, state.nets, zero, view.X, view.Y, view.L);
            const int* rec = enc.points.data() + enc.points[0];
            const int cnt = rec[1];
            const auto& graph = nt.rsmt;
            const int nodes = int(graph.size()) - 1;
            int root = 0;
            for (int i = 0; i < nodes; ++i)
                if (graph[i].size() == 1) { root = i; break; }
            ord.clear();
            parent.assign(nodes, -1);
            stack.assign(1, root);
            while (!stack.empty()) {
                const int v = stack.back();
                stack.pop_back();
                ord.push_back(v);
                for (auto it = graph[v].rbegin(); it != graph[v].rend(); ++it) {
                    if (*it == parent[v]) continue;
                    parent[*it] = v;
                    stack.push_back(*it);
                }
            }
            for (int k = 0; k < cnt; ++k) {
                P.coord.push_back(graph.back()[ord[k]]);
                for (int j = 0; j < 3; ++j) {
                    const int c = rec[2 + 6 * k + 3 + j];
                    P.child.push_back(c < 0 ? -1 : c / 6);
                }
            }
            P.size.push_back(cnt);
        }
    }
    for (const Part& P : parts) {
        for (int n : P.size) Z.node_off.push_back(Z.node_off.back() + n);
        Z.coord.insert(Z.coord.end(), P.coord.begin(), P.coord.end());
        Z.child.insert(Z.child.end(), P.child.begin(), P.child.end());
    }
    Z.t.node_off = Z.node_off.data();
    Z.t.coord = Z.coord.data();
    Z.t.child = Z.child.data();
    return Z;
}

// canonicalize_routes (zshape_topology.hpp:184-248) rewrites each net's route
// from that route alone, so contiguous ranges of nets go to host threads, each
// calling the reference's function with the offsets of its range (a net's
// words stay where the whole-array call would put them).
void canonicalize_parallel(cudb::RouterState& state, int count) {
    constexpr int kParts = 8;
    std::vector<std::exception_ptr> err(kParts);
#pragma omp parallel for num_threads(kParts) schedule(static, 1)
    for (int t = 0; t < kParts; ++t) {
        const int lo = int(int64_t(count) * t / kParts), hi = int(int64_t(count) * (t + 1) / kParts);
        if (lo >= hi) continue;
        try {
            const std::vector<int> offsets(state.pin_cnt_sum_cpu.begin() + lo, state.pin_cnt_sum_cpu.begin() + hi + 1);
            grotor::zshape::canonicalize_routes(hi - lo, state.device.X, state.device.Y, state.device.ROUTE_PER_PIN,
                                                offsets, state.routes_cpu.get());
        } catch (...) {
            err[t] = std::current_exception();
        }
    }
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

void route_ggr(cudb::RouterState& state, int32_t mode) {
    state.device.ROUTE_PER_PIN = 256;  // pipeline_ggr.hpp:9
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
    auto& nets = state.nets;
    const int count = int(nets.size());
    printf("ROUTING_STAGE_BEGIN stage=zshape nets=%d\n", count);  // pipeline_ggr.hpp:17
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    const auto topology_start = std::chrono::steady_clock::now();
#pragma omp parallel for num_threads(8)
    for (int i = 0; i < count; ++i) nets[i].construct_rsmt(state, true);
    phases.mark("flute");
    Trees F = flatten_trees(state);
    check(grb_build_topology(ctx, &F.t), ctx, "grb_build_topology");
    ZTrees Z = encode_trees(state);
    check(grb_upload_zshape(ctx, &Z.t), ctx, "grb_upload_zshape");
    phases.mark("topology");
    printf("TOPOLOGY_TIMING stage=zshape elapsed_ms=%.6f executor=grotor_b200\n",
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - topology_start).count());
    // pipeline_ggr.hpp:31-33: HPWL descending, larger id first on ties.
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return nets[a].hpwl == nets[b].hpwl ? a > b : nets[a].hpwl > nets[b].hpwl;
    });
    check(grb_set_stats(ctx, 0.0, initial_vias), ctx, "grb_set_stats");
    check(grb_set_wire_cost_mode(ctx, 1), ctx, "grb_set_wire_cost_mode");
    int32_t groups = 0, nb = 0;
    check(grb_plan_batches(ctx, order.data(), count, 1000000, state.batch_sparsity_override,
                           mode == GRB_MODE_PERSISTENT ? GRB_MODE_PERSISTENT : GRB_MODE_PLAIN, nullptr, &groups),
          ctx, "grb_plan_batches");
    std::vector<int32_t> bbox;
    for (const auto& nt : nets) { bbox.push_back(nt.minx); bbox.push_back(nt.maxx); bbox.push_back(nt.miny); bbox.push_back(nt.maxy); }
    check(grb_plan_bbox_batches(ctx, bbox.data(), 250, &nb), ctx, "grb_plan_bbox_batches");
    grb_stats st{};
    phases.mark("plan");
    const int zrc = grb_zshape_stage(ctx, mode, &st);
    if (zrc == GRB_ELIMIT) throw std::runtime_error(std::string("Z-shape DP failure or route storage overflow: ") + grb_last_error(ctx));
    check(zrc, ctx, "grb_zshape_stage");
    printf("BATCH_TIMING backend=grotor_b200 elapsed_ms=%.6f nets=%d batches=%d used_for_routing=1\n", st.batching_ms,
           count, nb);
    printf("DAG_TIMING stage=zshape batch_index=-1 elapsed_ms=%.6f nets=%d batches=%d executor=grotor_b200\n",
           st.dag_ms, count, nb);
    // pipeline_ggr.hpp:142-151: the reference's post-processing on the
    // downloaded routes, then the routes go back for the device writer.
    const size_t words = size_t(state.device.ROUTE_PER_PIN) * state.device.PIN_NUM + 1;
    // Only the words in use move (the post-processing and the writer read a
    // route below its count word), so the storage needs no clearing.
    state.routes_cpu.reset(new int[words]);
    check(grb_read_routes_used(ctx, state.routes_cpu.get()), ctx, "grb_read_routes_used");
    phases.mark("stage_download");
    const auto post_begin = std::chrono::steady_clock::now();
    const int promoted = grotor::zshape::promote_congested_segments(count, state.device.X, state.device.Y, state.device.L,
        state.device.ROUTE_PER_PIN, state.pin_cnt_sum_cpu, state.routes_cpu.get());
    phases.mark("postprocess_promote");
    canonicalize_parallel(state, count);
    printf("ZSHAPE_POSTPROCESS promoted_segments=%d elapsed_ms=%.6f\n", promoted,
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - post_begin).count());
    phases.mark("postprocess");
    check(grb_write_routes_used(ctx, state.routes_cpu.get()), ctx, "grb_write_routes_used");
    for (int i = 0; i < int(db::nets.size()); ++i)
        if (db::nets[i].pins.size() == 1) nets2output.push(i);
    graph::finish_nets(state, order);
    Output out{ctx};
    out.start(state);
    out.wait();
    phases.mark("output");
    printf("ROUTING_STAGE_END stage=zshape\n");  // pipeline_ggr.hpp:159
}

}  // namespace drop_in

int main(int argc, char** argv) {
    try {
        std::string cap, net, output, lut_dir = ".", executor = "persistent";
        if (argc < 7 || argc % 2 != 1)
            throw std::invalid_argument("Usage: grotor_grb_ggr -cap FILE -net FILE -out FILE [--lut-dir DIR] "
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
            drop_in::route_ggr(state, mode);
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
        fprintf(stderr, "grotor_grb_ggr error: %s\n", error.what());
        return EXIT_FAILURE;
    }
}
