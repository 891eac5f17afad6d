// Index builder: runs the ARTEA reference's own CPU builder on a vector file
// and writes the compacted graph as an HGRA v1 snapshot.
//
// The GPU router searches graphs; it does not build them. Graphs are produced
// exactly as the reference's quick start does (README.md "Quick Start";
// unit_tests/test_artea_graph.cpp:276-340):
//   artea_graph::factory_t::add_vertices (r-net insertion + per-layer refine)
//   -> hierarchical_graph_compactor_t::compact_graph (trim, CSR, centroid entry)
//   -> hierarchical_graph_file_manager_t::snapshot  (HGRA v1 wire format)
// with the build metric mapping of build_infra_dispatch
// (framework/type_context/infra_dispatcher.hpp:223-230): Euclidean graphs are
// built with true L2, cosine and dot keep their metric.
//
// This file is compiled against the reference headers where they lie plus the
// shim headers in index_build/shim (oneTBB subset, MKL VSL stub, termcolor,
// boost declarations); no reference source is copied.
//
// Usage:
//   artea_build_index --base BASE.fbin --metric euclidean|cosine|dot --out G.hgra
//       [--beta 2.0] [--tau-k 0] [--tau 1.5] [--l0 1.0] [--search-nn-qs 64]
//       [--ul-select-qs 100] [--bl-select-qs 100] [--ul-max 32] [--bl-max 64]
//       [--loops 15] [--triu 4] [--prefill 0.4] [--scale 1.10] [--shift 1.5]
//       [--shuffle 1] [--insert-on-l0 0]
// Prints one JSON line with build/compaction times and the level histogram.

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <artea/cpu/framework/type_context/default_context.hpp>

using namespace artea::cpu;

namespace {

struct Args {
    std::string base, out, metric = "euclidean";
    float beta = 2.0f, tau_k = 0.0f, tau = 1.5f, l0 = 1.0f;
    uint32_t search_nn_qs = 64, ul_select_qs = 100, bl_select_qs = 100, ul_max = 32, bl_max = 64;
    uint32_t loops = 15, triu = 4;
    float prefill = 0.4f, scale = 1.10f, shift = 1.5f;
    bool shuffle = true, insert_on_l0 = false;
};

Args parse(int argc, char** argv) {
    Args a;
    std::map<std::string, std::string> kv;
    for (int i = 1; i + 1 < argc; i += 2) kv[argv[i]] = argv[i + 1];
    if (argc % 2 == 0) throw std::invalid_argument("arguments must come in --key value pairs");
    auto f = [&](const char* k, float& v) { if (kv.count(k)) v = std::stof(kv[k]); };
    auto u = [&](const char* k, uint32_t& v) { if (kv.count(k)) v = static_cast<uint32_t>(std::stoul(kv[k])); };
    auto b = [&](const char* k, bool& v) { if (kv.count(k)) v = std::stoi(kv[k]) != 0; };
    if (kv.count("--base")) a.base = kv["--base"];
    if (kv.count("--out")) a.out = kv["--out"];
    if (kv.count("--metric")) a.metric = kv["--metric"];
    f("--beta", a.beta); f("--tau-k", a.tau_k); f("--tau", a.tau); f("--l0", a.l0);
    u("--search-nn-qs", a.search_nn_qs); u("--ul-select-qs", a.ul_select_qs);
    u("--bl-select-qs", a.bl_select_qs); u("--ul-max", a.ul_max); u("--bl-max", a.bl_max);
    u("--loops", a.loops); u("--triu", a.triu);
    f("--prefill", a.prefill); f("--scale", a.scale); f("--shift", a.shift);
    b("--shuffle", a.shuffle); b("--insert-on-l0", a.insert_on_l0);
    if (a.base.empty() || a.out.empty()) throw std::invalid_argument("--base and --out are required");
    return a;
}

vector_array_t load_fbin(const std::string& path) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("cannot open " + path);
    uint32_t hdr[2];
    if (std::fread(hdr, sizeof(uint32_t), 2, fp) != 2) throw std::runtime_error("short header in " + path);
    vector_array_t v(hdr[0], hdr[1]);
    const std::size_t total = std::size_t(hdr[0]) * hdr[1];
    if (total && std::fread(v.get_all(), sizeof(float), total, fp) != total) {
        std::fclose(fp);
        throw std::runtime_error("short payload in " + path);
    }
    std::fclose(fp);
    return v;
}

template <DistanceMetricsT Metric, vec_dim_t Dim>
int build(const Args& a, const vector_array_t& base) {
    dist_func_t<Metric, Dim> build_dist;
    artea_graph::rgraph_config_t<Metric, Dim> rgraph_cfg(
        a.beta, a.tau_k, a.tau, a.l0, a.search_nn_qs, a.ul_select_qs, a.bl_select_qs, a.ul_max, a.bl_max);
    artea_graph::propagate_config_t<Metric, Dim> propagate_cfg(a.loops, a.triu, a.prefill);
    artea_graph::pruning_config_t<Metric, Dim> pruning_cfg(a.scale, a.shift, a.l0);

    const auto n = base.get_num_vecs();
    auto t0 = std::chrono::steady_clock::now();
    auto graph = std::make_unique<artea_graph::index_t<Metric, Dim>>(n, rgraph_cfg, propagate_cfg, pruning_cfg);
    artea_graph::factory_t<Metric, Dim>::add_vertices(
        *graph, base.extract_subset(0, n), build_dist, a.insert_on_l0, a.shuffle);
    auto t1 = std::chrono::steady_clock::now();
    auto compact = hierarchical_graph_compactor_t::compact_graph(graph->get_hierarchical_graph(), base, build_dist);
    auto t2 = std::chrono::steady_clock::now();
    graph.reset();
    hierarchical_graph_file_manager_t::snapshot(compact, a.out);

    const auto top = compact.top_occupied_level_id();
    std::string hist = "[";
    if (top != compact::hierarchical_graph_t::invalid_level_id) {
        for (uint32_t h = 0; h <= top; ++h) {
            hist += (h ? "," : "") + std::to_string(compact.get_vids_with_highest_level(h).size());
        }
    }
    hist += "]";
    const double build_s = std::chrono::duration<double>(t1 - t0).count();
    const double compact_s = std::chrono::duration<double>(t2 - t1).count();
    std::printf("{\"n\": %u, \"dim\": %u, \"metric\": \"%s\", \"build_s\": %.3f, \"compact_s\": %.3f, "
                "\"top_level\": %d, \"entry\": %u, \"n_nbrs\": %zu, \"vertices_by_highest_level\": %s, "
                "\"threads\": %d}\n",
                n, Dim, a.metric.c_str(), build_s, compact_s,
                top == compact::hierarchical_graph_t::invalid_level_id ? -1 : int(top),
                compact.entry_point_vid(), compact.neighbor_ids().size(), hist.c_str(),
                tbb::this_task_arena::max_concurrency());
    return 0;
}

template <DistanceMetricsT Metric>
int dispatch_dim(const Args& a, const vector_array_t& base) {
    switch (base.get_vec_dim()) {
        case 16: return build<Metric, 16>(a, base);
        case 96: return build<Metric, 96>(a, base);
        case 128: return build<Metric, 128>(a, base);
        case 960: return build<Metric, 960>(a, base);
        default: break;
    }
    throw std::invalid_argument("unsupported padded dim " + std::to_string(base.get_vec_dim()));
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const Args a = parse(argc, argv);
        const vector_array_t base = load_fbin(a.base);
        if (a.metric == "euclidean" || a.metric == "l2") return dispatch_dim<DistanceMetricsT::EUCLIDEAN>(a, base);
        if (a.metric == "cosine") return dispatch_dim<DistanceMetricsT::COSINE>(a, base);
        if (a.metric == "dot") return dispatch_dim<DistanceMetricsT::DOT>(a, base);
        throw std::invalid_argument("unknown metric " + a.metric);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "artea_build_index: %s\n", e.what());
        return 2;
    }
}
