// Drop-in check: the same calls on the reference's CPU router
// (hierarchical_graph_router_t<Metric, Dim>) and on
// artea::cuda::HierarchicalGraphRouter<router_traits_t<Metric, Dim>> must
// return identical knn_results_t (EXACT mode). The graph is the reference's
// own compact::hierarchical_graph_t restored from an HGRA snapshot.
//
// usage: test_dropin GRAPH.hgra BASE.fbin QUERIES.fbin METRIC TOPK QUEUE
//        test_dropin --cpu-only     (constructor contract only; no GPU)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>
#include <stdexcept>
#include <string>

#include <artea/cpu/framework/type_context/default_context.hpp>
#include <artea/cpu/index/exact_artea/configs.hpp>
#include <artea_b200/hierarchical_graph_router.hpp>

using namespace artea::cpu;

namespace {

vector_array_t load_fbin(const char* path) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) throw std::runtime_error(std::string("cannot open ") + path);
    uint32_t hdr[2];
    if (std::fread(hdr, 4, 2, fp) != 2) throw std::runtime_error("short header");
    vector_array_t v(hdr[0], hdr[1]);
    const size_t total = size_t(hdr[0]) * hdr[1];
    if (total && std::fread(v.get_all(), 4, total, fp) != total) throw std::runtime_error("short payload");
    std::fclose(fp);
    return v;
}

template <typename R>
bool same(const R& a, const R& b, const char* what) {
    if (a.size() != b.size() || (a.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(a[0])) != 0)) {
        std::printf("MISMATCH %s (%zu vs %zu entries)\n", what, a.size(), b.size());
        return false;
    }
    return true;
}

using rgraph_config_t = index_traits_t::exact_artea::rgraph_config_t;
using pruning_config_t = index_traits_t::exact_artea::pruning_config_t;

// Per-level thresholds in the shape of an RGraphConfig (early_stop_threshold(h, pruning)).
struct TableConfig {
    std::vector<float> t;
    auto early_stop_threshold(uint32_t h, const pruning_config_t&) const -> float { return t.at(h); }
};

// enable_early_stop=true through the explicit-config overloads
// (hierarchical_graph_router.hpp:176-190, :308-319): identical results, and
// the same std::overflow_error for a threshold that squares past FLT_MAX.
template <DistanceMetricsT M, typename Cpu, typename Gpu>
bool early_stop_checks(const Cpu& cpu, const Gpu& gpu, const compact::hierarchical_graph_t& g,
                       const vector_array_t& base, const vector_array_t& queries) {
    bool ok = true;
    const pruning_config_t pruning(2, 0);
    const rgraph_config_t cfg(2, 0, 0, 1, 4, 4, 4, 4, 4);   // test_router_early_stop.cpp:52-53
    ok &= same(cpu.template batch_query<false, true>(queries, g, cfg, pruning),
               gpu.template batch_query<false, true>(queries, g, cfg, pruning), "batch_query early stop (config)");
    const auto top = g.top_occupied_level_id();
    if (top == compact::hierarchical_graph_t::invalid_level_id || top == 0) return ok;
    // Thresholds that stop about half the walks: the median query-to-entry
    // distance in configuration (L2) units.
    std::vector<float> d;
    for (uint32_t i = 0; i < queries.get_num_vecs(); ++i) {
        double s = 0;
        for (uint32_t j = 0; j < base.get_vec_dim(); ++j) {
            const double x = double(queries.get(i)[j]) - double(base.get(g.entry_point_vid())[j]);
            s += x * x;
        }
        d.push_back(static_cast<float>(std::sqrt(s)));
    }
    std::sort(d.begin(), d.end());
    const TableConfig table{std::vector<float>(top + 1, d[d.size() / 2])};
    ok &= same(cpu.template batch_query<false, true>(queries, g, table, pruning),
               gpu.template batch_query<false, true>(queries, g, table, pruning), "batch_query early stop (table)");
    for (uint32_t i = 0; i < queries.get_num_vecs() && i < 8; ++i)
        ok &= same(cpu.template query<false, true>(queries.get(i), g, table, pruning),
                   gpu.template query<false, true>(queries.get(i), g, table, pruning), "query early stop");
    if constexpr (M == DistanceMetricsT::EUCLIDEAN_SQR) {
        const TableConfig huge{std::vector<float>(top + 1, 1e20f)};
        int thrown = 0;
        try { (void)cpu.template batch_query<false, true>(queries, g, huge, pruning); }
        catch (const std::overflow_error&) { ++thrown; }
        try { (void)gpu.template batch_query<false, true>(queries, g, huge, pruning); }
        catch (const std::overflow_error&) { ++thrown; }
        if (thrown != 2) {
            std::printf("MISMATCH overflow_error (%d of 2 threw)\n", thrown);
            ok = false;
        }
    }
    return ok;
}

template <DistanceMetricsT M, vec_dim_t D>
int run(const char* path, const compact::hierarchical_graph_t& g, const vector_array_t& base,
        const vector_array_t& queries, uint32_t topk, uint32_t queue) {
    dist_func_t<M, D> dist;
    hierarchical_graph_router_t<M, D> cpu(base, dist, topk, queue);
    cpu.initialize();
    artea::cuda::HierarchicalGraphRouter<router_traits_t<M, D>> gpu(base, dist, topk, queue);
    gpu.initialize();
    bool ok = true;
    const auto a = cpu.template batch_query<false>(queries, g);
    const auto b = gpu.template batch_query<false>(queries, g);
    ok &= same(a, b, "batch_query");
    const auto c = cpu.template batch_query_l0_only<false>(queries, g);
    const auto d = gpu.template batch_query_l0_only<false>(queries, g);
    ok &= same(c, d, "batch_query_l0_only");
    for (uint32_t i = 0; i < queries.get_num_vecs() && i < 8; ++i) {
        ok &= same(cpu.template query<false>(queries.get(i), g), gpu.template query<false>(queries.get(i), g),
                   "query");
    }
    ok &= early_stop_checks<M>(cpu, gpu, g, base, queries);
    // back to enable_early_stop=false on the same routers
    ok &= same(cpu.template batch_query<false>(queries, g), gpu.template batch_query<false>(queries, g),
               "batch_query after early stop");
    // A graph restored where a destroyed one lived is searched as itself, not
    // as the device copy of its predecessor: an empty graph, then the snapshot
    // restored into the same storage.
    {
        alignas(compact::hierarchical_graph_t) unsigned char slot[sizeof(compact::hierarchical_graph_t)];
        auto* first = new (slot) compact::hierarchical_graph_t(0, g.ul_max_nbr_size(), g.bl_max_nbr_size(), 0,
                                                                std::vector<std::size_t>{0});
        ok &= same(cpu.template batch_query<false>(queries, *first), gpu.template batch_query<false>(queries, *first),
                   "batch_query on an empty graph");
        std::destroy_at(first);
        auto* second = new (slot) compact::hierarchical_graph_t(hierarchical_graph_file_manager_t::restore(path));
        ok &= same(cpu.template batch_query<false>(queries, *second),
                   gpu.template batch_query<false>(queries, *second), "batch_query on a graph at a reused address");
        std::destroy_at(second);
    }
    std::printf("%s %zu batch entries compared\n", ok ? "OK" : "FAIL", a.size());
    return ok ? 0 : 1;
}

template <DistanceMetricsT M>
int by_dim(const char* path, const compact::hierarchical_graph_t& g, const vector_array_t& base,
           const vector_array_t& q, uint32_t k, uint32_t L) {
    switch (base.get_vec_dim()) {
        case 16: return run<M, 16>(path, g, base, q, k, L);
        case 96: return run<M, 96>(path, g, base, q, k, L);
        case 128: return run<M, 128>(path, g, base, q, k, L);
        case 960: return run<M, 960>(path, g, base, q, k, L);
        default: throw std::runtime_error("unsupported dim");
    }
}

int cpu_only() {
    // The constructor contract of hierarchical_graph_router.hpp:104-108:
    // queue < topk throws std::runtime_error, in both routers.
    vector_array_t base(4, 16);
    dist_func_t<DistanceMetricsT::EUCLIDEAN_SQR, 16> dist;
    int thrown = 0;
    try {
        hierarchical_graph_router_t<DistanceMetricsT::EUCLIDEAN_SQR, 16> r(base, dist, 10, 5);
    } catch (const std::runtime_error&) { ++thrown; }
    try {
        artea::cuda::HierarchicalGraphRouter<router_traits_t<DistanceMetricsT::EUCLIDEAN_SQR, 16>> r(base, dist, 10, 5);
    } catch (const std::runtime_error&) { ++thrown; }
    std::printf("%s constructor contract (%d of 2 threw)\n", thrown == 2 ? "OK" : "FAIL", thrown);
    return thrown == 2 ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc == 2 && std::strcmp(argv[1], "--cpu-only") == 0) return cpu_only();
        if (argc != 7) {
            std::fprintf(stderr, "usage: %s GRAPH.hgra BASE.fbin QUERIES.fbin METRIC TOPK QUEUE\n", argv[0]);
            return 2;
        }
        const auto g = hierarchical_graph_file_manager_t::restore(argv[1]);
        const auto base = load_fbin(argv[2]);
        const auto queries = load_fbin(argv[3]);
        const int metric = std::atoi(argv[4]);
        const uint32_t k = static_cast<uint32_t>(std::atoi(argv[5]));
        const uint32_t L = static_cast<uint32_t>(std::atoi(argv[6]));
        switch (metric) {
            case 0: return by_dim<DistanceMetricsT::EUCLIDEAN_SQR>(argv[1], g, base, queries, k, L);
            case 1: return by_dim<DistanceMetricsT::EUCLIDEAN>(argv[1], g, base, queries, k, L);
            case 2: return by_dim<DistanceMetricsT::COSINE>(argv[1], g, base, queries, k, L);
            case 3: return by_dim<DistanceMetricsT::DOT>(argv[1], g, base, queries, k, L);
            default: throw std::runtime_error("unknown metric");
        }
    } catch (const std::exception& e) {
        std::printf("ERROR %s\n", e.what());
        return 3;
    }
}
