// ORACLE — test infrastructure only. C entry points around the ARTEA
// reference's own CPU router, compiled from the reference headers where they
// lie (see oracle/Makefile) into oracle/_ref/libartea_ref.so. Used by tests/
// to pin the C restatement (artea_oracle.c) and by bench.py's CPU baseline
// arm; the product never links it.
//
// The router is the reference's hierarchical_graph_router_t<Metric, Dim>
// (framework/type_context/default_context.hpp:158) over a compact graph
// restored with hierarchical_graph_file_manager_t::restore
// (index/persistence/hierarchical_graph_file_manager.hpp:152), queried with
// batch_query<RandomSeeding=false> (router/hierarchical_graph_router.hpp:293-304).

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <tbb/global_control.h>

#include <artea/cpu/framework/type_context/default_context.hpp>

using namespace artea::cpu;

namespace {

thread_local std::string g_last_error;

struct RefIndex {
    compact::hierarchical_graph_t graph;
    vector_array_t vecs;
};

vector_array_t copy_rows(const float* src, uint32_t n, uint32_t dim) {
    vector_array_t v(n, dim);
    if (n) std::memcpy(v.get_all(), src, sizeof(float) * std::size_t(n) * dim);
    return v;
}

// Distance functor that counts calls in a thread-local counter, in the manner
// of unit_tests/test_router_early_stop.cpp:43-50.
thread_local uint64_t t_dist_calls = 0;

template <DistanceMetricsT Metric, vec_dim_t Dim>
struct CountingComputer : ComputerTraits<base_traits_t, Metric, Dim> {
    struct dist_func_t {
        auto operator()(const float* a, const float* b) const -> float {
            ++t_dist_calls;
            return typename ComputerTraits<base_traits_t, Metric, Dim>::dist_func_t{}(a, b);
        }
    };
};

template <DistanceMetricsT Metric, vec_dim_t Dim>
int run(RefIndex& idx, const float* queries, uint32_t nq, uint32_t topk, uint32_t queue,
        int l0_only, uint64_t* out, double* seconds, uint64_t* dist_calls) {
    vector_array_t qv = copy_rows(queries, nq, Dim);
    if (dist_calls) {
        // Counting variant: per-query query() calls, sequential.
        using RT = RouterTraits<CountingComputer<Metric, Dim>, index_traits_t, false>;
        typename RT::dist_func_t dist;
        typename RT::hierarchical_graph_router_t router(idx.vecs, dist, topk, queue);
        router.initialize();
        const auto t0 = std::chrono::steady_clock::now();
        for (uint32_t i = 0; i < nq; ++i) {
            t_dist_calls = 0;
            auto r = l0_only ? router.template query_l0_only<false>(qv.get(i), idx.graph)
                             : router.template query<false>(qv.get(i), idx.graph);
            dist_calls[i] = t_dist_calls;
            for (uint32_t j = 0; j < topk; ++j) {
                const auto e = j < r.size() ? r[j] : RT::candidate_entry_t::make_invalid_entry();
                std::memcpy(out + std::size_t(i) * topk + j, &e, sizeof(uint64_t));
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    }
    dist_func_t<Metric, Dim> dist;
    hierarchical_graph_router_t<Metric, Dim> router(idx.vecs, dist, topk, queue);
    router.initialize();
    const auto t0 = std::chrono::steady_clock::now();
    auto res = l0_only ? router.template batch_query_l0_only<false>(qv, idx.graph)
                       : router.template batch_query<false>(qv, idx.graph);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    static_assert(sizeof(res[0]) == sizeof(uint64_t));
    std::memcpy(out, res.data(), sizeof(uint64_t) * res.size());
    return 0;
}

// Per-level thresholds handed to the reference's enable_early_stop overloads
// (hierarchical_graph_router.hpp:176-190, :308-319) in the shape of the
// configuration they read (RGraphConfig::early_stop_threshold(h, pruning)).
struct TableConfig {
    const float* thr;
    uint32_t n;
    auto early_stop_threshold(uint32_t h, const TableConfig&) const -> float {
        return h < n ? thr[h] : std::numeric_limits<float>::quiet_NaN();
    }
};

template <DistanceMetricsT Metric, vec_dim_t Dim>
int run_early_stop(RefIndex& idx, const float* queries, uint32_t nq, uint32_t topk, uint32_t queue,
                   const TableConfig& cfg, uint64_t* out, uint64_t* dist_calls) {
    vector_array_t qv = copy_rows(queries, nq, Dim);
    using RT = RouterTraits<CountingComputer<Metric, Dim>, index_traits_t, false>;
    typename RT::dist_func_t dist;
    typename RT::hierarchical_graph_router_t router(idx.vecs, dist, topk, queue);
    router.initialize();
    const auto batch = router.template batch_query<false, true>(qv, idx.graph, cfg, cfg);
    std::memcpy(out, batch.data(), sizeof(uint64_t) * batch.size());
    if (dist_calls) {
        for (uint32_t i = 0; i < nq; ++i) {
            t_dist_calls = 0;
            auto r = router.template query<false, true>(qv.get(i), idx.graph, cfg, cfg);
            dist_calls[i] = t_dist_calls;
            for (uint32_t j = 0; j < topk; ++j) {
                const auto e = j < r.size() ? r[j] : RT::candidate_entry_t::make_invalid_entry();
                uint64_t w;
                std::memcpy(&w, &e, sizeof(w));
                if (w != out[std::size_t(i) * topk + j])
                    throw std::logic_error("reference query and batch_query disagree under early stop");
            }
        }
    }
    return 0;
}

template <DistanceMetricsT Metric>
int by_dim_es(RefIndex& idx, const float* q, uint32_t nq, uint32_t k, uint32_t L, const TableConfig& cfg,
              uint64_t* out, uint64_t* calls) {
    switch (idx.vecs.get_vec_dim()) {
        case 16: return run_early_stop<Metric, 16>(idx, q, nq, k, L, cfg, out, calls);
        case 96: return run_early_stop<Metric, 96>(idx, q, nq, k, L, cfg, out, calls);
        case 128: return run_early_stop<Metric, 128>(idx, q, nq, k, L, cfg, out, calls);
        case 960: return run_early_stop<Metric, 960>(idx, q, nq, k, L, cfg, out, calls);
        default: break;
    }
    throw std::invalid_argument("unsupported padded dim " + std::to_string(idx.vecs.get_vec_dim()));
}

template <DistanceMetricsT Metric>
int by_dim(RefIndex& idx, const float* q, uint32_t nq, uint32_t k, uint32_t L, int l0_only, uint64_t* out,
           double* s, uint64_t* calls) {
    switch (idx.vecs.get_vec_dim()) {
        case 16: return run<Metric, 16>(idx, q, nq, k, L, l0_only, out, s, calls);
        case 96: return run<Metric, 96>(idx, q, nq, k, L, l0_only, out, s, calls);
        case 128: return run<Metric, 128>(idx, q, nq, k, L, l0_only, out, s, calls);
        case 960: return run<Metric, 960>(idx, q, nq, k, L, l0_only, out, s, calls);
        default: break;
    }
    throw std::invalid_argument("unsupported padded dim " + std::to_string(idx.vecs.get_vec_dim()));
}

// bruteforce_router_t<Metric, Dim>::batch_query (router/bruteforce_router.hpp:130-160)
// or, with subset != null, its subset overload (:164-190). out: nq*topk words.
template <DistanceMetricsT Metric, vec_dim_t Dim>
int run_bruteforce(RefIndex& idx, const float* queries, uint32_t nq, uint32_t topk, const uint32_t* subset,
                   uint32_t n_subset, uint64_t* out) {
    vector_array_t qv = copy_rows(queries, nq, Dim);
    dist_func_t<Metric, Dim> dist;
    bruteforce_router_t<Metric, Dim> router(idx.vecs, dist, topk);
    router.initialize();
    const auto res = subset ? router.batch_query(qv, std::span<const uint32_t>(subset, n_subset))
                            : router.batch_query(qv);
    std::memcpy(out, res.data(), sizeof(uint64_t) * res.size());
    return 0;
}

template <DistanceMetricsT Metric>
int by_dim_bf(RefIndex& idx, const float* q, uint32_t nq, uint32_t k, const uint32_t* s, uint32_t ns,
              uint64_t* out) {
    switch (idx.vecs.get_vec_dim()) {
        case 16: return run_bruteforce<Metric, 16>(idx, q, nq, k, s, ns, out);
        case 96: return run_bruteforce<Metric, 96>(idx, q, nq, k, s, ns, out);
        case 128: return run_bruteforce<Metric, 128>(idx, q, nq, k, s, ns, out);
        case 960: return run_bruteforce<Metric, 960>(idx, q, nq, k, s, ns, out);
        default: break;
    }
    throw std::invalid_argument("unsupported padded dim " + std::to_string(idx.vecs.get_vec_dim()));
}

}  // namespace

extern "C" {


const char* artea_ref_last_error() { return g_last_error.c_str(); }

void* artea_ref_open(const char* hgra_path, const float* vecs, uint32_t n, uint32_t dim) {
    try {
        auto g = hierarchical_graph_file_manager_t::restore(hgra_path);
        return new RefIndex{std::move(g), copy_rows(vecs, n, dim)};
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return nullptr;
    }
}

void artea_ref_close(void* h) { delete static_cast<RefIndex*>(h); }

// The reference's restore of a snapshot in the compact graph's own arrays
// (index/compact_structure/hierarchical_graph.hpp:46-49, 96-101): sizes[0..3]
// = vertices, groups, offsets over all groups, neighbour ids; with non-null
// arrays also vertex_info (highest level, local vid per vertex; invalid
// levels as 0xFFFFFFFF), the groups' offsets concatenated in level order and
// the neighbour ids. Returns 0, or -1 on an error.
int artea_ref_restore_layout(const char* hgra_path, uint64_t* sizes, uint32_t* vertex_info, uint64_t* offsets,
                             uint32_t* nbrs) {
    try {
        auto g = hierarchical_graph_file_manager_t::restore(hgra_path);
        const uint64_t n = g.get_num_vertices();
        const auto top = g.top_occupied_level_id();
        using level_t = std::remove_cv_t<decltype(top)>;
        const uint64_t groups = n == 0 ? 0 : static_cast<uint64_t>(top) + 1;
        uint64_t total = 0;
        for (uint64_t h = 0; h < groups; ++h) total += g.get_nbr_offsets(static_cast<level_t>(h)).size();
        const auto ids = g.neighbor_ids();
        sizes[0] = n;
        sizes[1] = groups;
        sizes[2] = total;
        sizes[3] = ids.size();
        if (!vertex_info) return 0;
        for (uint64_t v = 0; v < n; ++v) {
            const auto& info = g.get_vertex_info(static_cast<uint32_t>(v));
            const bool none = info.highest_level == std::numeric_limits<level_t>::max();
            vertex_info[2 * v] = none ? 0xFFFFFFFFu : static_cast<uint32_t>(info.highest_level);
            vertex_info[2 * v + 1] = static_cast<uint32_t>(info.local_vid);
        }
        uint64_t at = 0;
        for (uint64_t h = 0; h < groups; ++h) {
            const auto off = g.get_nbr_offsets(static_cast<level_t>(h));
            std::memcpy(offsets + at, off.data(), sizeof(uint64_t) * off.size());
            at += off.size();
        }
        if (!ids.empty()) std::memcpy(nbrs, ids.data(), sizeof(uint32_t) * ids.size());
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Seconds taken by hierarchical_graph_file_manager_t::restore of the
// snapshot alone (index/persistence/hierarchical_graph_file_manager.hpp:152),
// the reference's way from an HGRA file to a searchable compact graph; the
// number of vertices restored, or -1 on an error.
long long artea_ref_restore_seconds(const char* hgra_path, double* seconds) {
    try {
        const auto t0 = std::chrono::steady_clock::now();
        auto g = hierarchical_graph_file_manager_t::restore(hgra_path);
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return static_cast<long long>(g.get_num_vertices());
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// metric: 0 EUCLIDEAN_SQR, 1 EUCLIDEAN, 2 COSINE, 3 DOT. out: nq*topk words.
// threads > 0 caps the worker count (tbb::global_control); dist_calls, if not
// null, switches to sequential per-query calls with a counting distance.
int artea_ref_batch_query(void* h, const float* queries, uint32_t nq, uint32_t topk, uint32_t queue,
                          int metric, int l0_only, int threads, uint64_t* out, double* seconds,
                          uint64_t* dist_calls) {
    try {
        auto& idx = *static_cast<RefIndex*>(h);
        std::unique_ptr<tbb::global_control> limit;
        if (threads > 0)
            limit = std::make_unique<tbb::global_control>(tbb::global_control::max_allowed_parallelism, threads);
        switch (metric) {
            case 0: return by_dim<DistanceMetricsT::EUCLIDEAN_SQR>(idx, queries, nq, topk, queue, l0_only, out, seconds, dist_calls);
            case 1: return by_dim<DistanceMetricsT::EUCLIDEAN>(idx, queries, nq, topk, queue, l0_only, out, seconds, dist_calls);
            case 2: return by_dim<DistanceMetricsT::COSINE>(idx, queries, nq, topk, queue, l0_only, out, seconds, dist_calls);
            case 3: return by_dim<DistanceMetricsT::DOT>(idx, queries, nq, topk, queue, l0_only, out, seconds, dist_calls);
            default: throw std::invalid_argument("unknown metric");
        }
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// batch_query<RandomSeeding=false, enable_early_stop=true> with per-level
// configuration thresholds cfg[0, n_levels). Returns 0, -1 on an error, -2
// when the reference throws std::overflow_error (threshold not representable).
int artea_ref_batch_query_early_stop(void* h, const float* queries, uint32_t nq, uint32_t topk, uint32_t queue,
                                     int metric, const float* cfg, uint32_t n_levels, uint64_t* out,
                                     uint64_t* dist_calls) {
    try {
        auto& idx = *static_cast<RefIndex*>(h);
        const TableConfig c{cfg, n_levels};
        switch (metric) {
            case 0: return by_dim_es<DistanceMetricsT::EUCLIDEAN_SQR>(idx, queries, nq, topk, queue, c, out, dist_calls);
            case 1: return by_dim_es<DistanceMetricsT::EUCLIDEAN>(idx, queries, nq, topk, queue, c, out, dist_calls);
            case 2: return by_dim_es<DistanceMetricsT::COSINE>(idx, queries, nq, topk, queue, c, out, dist_calls);
            case 3: return by_dim_es<DistanceMetricsT::DOT>(idx, queries, nq, topk, queue, c, out, dist_calls);
            default: throw std::invalid_argument("unknown metric");
        }
    } catch (const std::overflow_error& e) {
        g_last_error = e.what();
        return -2;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int artea_ref_bruteforce(void* h, const float* queries, uint32_t nq, uint32_t topk, int metric,
                                    const uint32_t* subset, uint32_t n_subset, uint64_t* out) {
    try {
        auto& idx = *static_cast<RefIndex*>(h);
        switch (metric) {
            case 0: return by_dim_bf<DistanceMetricsT::EUCLIDEAN_SQR>(idx, queries, nq, topk, subset, n_subset, out);
            case 1: return by_dim_bf<DistanceMetricsT::EUCLIDEAN>(idx, queries, nq, topk, subset, n_subset, out);
            case 2: return by_dim_bf<DistanceMetricsT::COSINE>(idx, queries, nq, topk, subset, n_subset, out);
            case 3: return by_dim_bf<DistanceMetricsT::DOT>(idx, queries, nq, topk, subset, n_subset, out);
            default: throw std::invalid_argument("unknown metric");
        }
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// The reference SIMD distance on one pair (utils/simd_distance.hpp:64-79).
float artea_ref_distance(int metric, const float* a, const float* b, uint32_t dim) {
    auto go = [&]<DistanceMetricsT M>() -> float {
        switch (dim) {
            case 16: return dist_func_t<M, 16>{}(a, b);
            case 96: return dist_func_t<M, 96>{}(a, b);
            case 128: return dist_func_t<M, 128>{}(a, b);
            case 960: return dist_func_t<M, 960>{}(a, b);
            default: return std::numeric_limits<float>::quiet_NaN();
        }
    };
    switch (metric) {
        case 0: return go.template operator()<DistanceMetricsT::EUCLIDEAN_SQR>();
        case 1: return go.template operator()<DistanceMetricsT::EUCLIDEAN>();
        case 2: return go.template operator()<DistanceMetricsT::COSINE>();
        case 3: return go.template operator()<DistanceMetricsT::DOT>();
        default: return std::numeric_limits<float>::quiet_NaN();
    }
}

int artea_ref_max_threads() { return tbb::this_task_arena::max_concurrency(); }

}  // extern "C"
