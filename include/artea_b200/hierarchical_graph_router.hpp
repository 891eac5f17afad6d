// artea::cuda::HierarchicalGraphRouter — drop-in for the reference router.
//
// Same template and call surface as the CPU router
// (include/artea/cpu/router/hierarchical_graph_router.hpp:66-430, reached as
// hierarchical_graph_router_t<Metric, Dim>, framework/type_context/default_context.hpp:158):
//
//   artea::cuda::HierarchicalGraphRouter<router_traits_t<Metric, Dim>> r(base_vecs, dist, topk, queue);
//   r.initialize();
//   knn_results_t res = r.batch_query</*RandomSeeding=*/false>(query_vecs, compact_hg);
//
// Header-only; it depends on the reference only through the traits and graph
// types it is instantiated with, and on libartea_gpu.so through the C-ABI of
// include/artea_gpu.h. The first batch_query with a graph uploads the graph and
// base_vecs (the router keeps a const reference to base_vecs, as the reference
// does, router/vector_router.hpp:46,63-69) and later calls reuse the device
// copy, keyed by the graph's address and checked against a fingerprint of its
// sizes, storage and a sample of its contents, so a graph restored where a
// destroyed one lived is uploaded afresh. Errors surface as std::runtime_error
// (the reference's ARTEA_ERROR, common/logger.hpp:97-99,149).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../artea_gpu.h"

namespace artea {
namespace cuda {

namespace detail {

inline void check(int status, const char* what) {
    if (status != ARTEA_GPU_OK) {
        throw std::runtime_error(std::string(what) + ": " + artea_gpu_last_error());
    }
}

// DistanceMetricsT of the traits -> artea_gpu_metric (simd_distance.hpp:64-79).
template <typename RouterTraitsT>
constexpr int metric_code() {
    using M = typename RouterTraitsT::distance_metrics_t;
    constexpr M m = RouterTraitsT::distance_metrics;
    if constexpr (m == M::EUCLIDEAN_SQR) return ARTEA_GPU_EUCLIDEAN_SQR;
    else if constexpr (m == M::EUCLIDEAN) return ARTEA_GPU_EUCLIDEAN;
    else if constexpr (m == M::COSINE) return ARTEA_GPU_COSINE;
    else return ARTEA_GPU_DOT;
}

}  // namespace detail

/** Options beyond the reference's ctor: distance mode (EXACT reproduces the
 *  reference bit for bit), schedule and device. */
struct RouterOptions {
    int mode = ARTEA_GPU_MODE_EXACT;
    int schedule = ARTEA_GPU_SCHEDULE_AUTO;
    int device = 0;
};

template <typename RouterTraitsT>
class HierarchicalGraphRouter {
public:
    using vertex_num_t = typename RouterTraitsT::vertex_num_t;
    using vertex_id_t = typename RouterTraitsT::vertex_id_t;
    using vec_ele_t = typename RouterTraitsT::vec_ele_t;
    using dist_func_t = typename RouterTraitsT::dist_func_t;
    using vector_array_t = typename RouterTraitsT::vector_array_t;
    using query_vecs_t = typename RouterTraitsT::query_vecs_t;
    using candidate_entry_t = typename RouterTraitsT::candidate_entry_t;
    using knn_results_t = typename RouterTraitsT::knn_results_t;

    static_assert(sizeof(candidate_entry_t) == 8, "results are 8-byte CandidateEntry words");
    static_assert(std::is_same_v<vec_ele_t, float>, "the GPU router searches FP32 vectors");
    static_assert(RouterTraitsT::vec_dim % 16 == 0, "Dim must be the SIMD-padded dimension (multiple of 16)");

    HierarchicalGraphRouter(const vector_array_t& base_vecs, const dist_func_t& dist_func, const uint32_t topk,
                            const vertex_num_t candidate_queue_size = 16, RouterOptions opts = {})
        : _vecs(base_vecs), _dist(dist_func), _topk(topk), _queue(candidate_queue_size), _opts(opts),
          _state(std::make_shared<State>()) {
        // hierarchical_graph_router.hpp:104-108
        if (candidate_queue_size < topk) {
            throw std::runtime_error("candidate_queue_size (" + std::to_string(candidate_queue_size) +
                                     ") must be >= topk (" + std::to_string(topk) + ")");
        }
    }

    /** hierarchical_graph_router.hpp:114-117. Checks that a device is usable;
     *  device state is created per graph on first use. */
    auto initialize() -> void {
        int n = 0;
        detail::check(artea_gpu_device_count(&n), "artea_gpu_device_count");
        if (_opts.device >= n) throw std::runtime_error("CUDA device not available");
    }

    /** batch_query<RandomSeeding, enable_early_stop>(query_vecs, graph)
     *  (hierarchical_graph_router.hpp:293-349): nq*topk entries, row-major,
     *  invalid-filled past each query's results. With enable_early_stop the
     *  graph must carry its configurations, as in the reference (:176-182). */
    template <bool RandomSeeding = false, bool enable_early_stop = false, typename HierarchicalGraphT>
    auto batch_query(const query_vecs_t& query_vecs, const HierarchicalGraphT& hier_graph) const -> knn_results_t {
        static_assert(!RandomSeeding, "the GPU router seeds from the graph's entry point (RandomSeeding=false)");
        static_assert(HierarchicalGraphT::is_compacted, "the GPU router searches compact graphs");
        if constexpr (enable_early_stop) {
            static_assert(requires { hier_graph.rgraph_config(); hier_graph.pruning_config(); },
                          "Early stopping on a bare graph requires explicit rgraph and pruning configs");
            return batch_query<RandomSeeding, true>(query_vecs, hier_graph, hier_graph.rgraph_config(),
                                                    hier_graph.pruning_config());
        } else {
            return _run(query_vecs.get_all(), query_vecs.get_num_vecs(), hier_graph, false, {});
        }
    }

    /** The explicit-config overload (hierarchical_graph_router.hpp:308-319):
     *  with enable_early_stop, the greedy walk on level h >= 1 stops once its
     *  cursor is within rgraph_config.early_stop_threshold(h, pruning_config),
     *  evaluated once per level per call (:388-408; squared for EUCLIDEAN_SQR
     *  by the library). Throws std::overflow_error when a threshold is not
     *  representable in query distance units. Without it the configs are not
     *  read. */
    template <bool RandomSeeding = false, bool enable_early_stop = false, typename HierarchicalGraphT,
              typename RGraphConfigT, typename PruningConfigT>
    auto batch_query(const query_vecs_t& query_vecs, const HierarchicalGraphT& hier_graph,
                     const RGraphConfigT& rgraph_config, const PruningConfigT& pruning_config) const
        -> knn_results_t {
        static_assert(!RandomSeeding, "the GPU router seeds from the graph's entry point (RandomSeeding=false)");
        static_assert(HierarchicalGraphT::is_compacted, "the GPU router searches compact graphs");
        if constexpr (enable_early_stop) {
            return _run(query_vecs.get_all(), query_vecs.get_num_vecs(), hier_graph, false,
                        _config_thresholds(hier_graph, rgraph_config, pruning_config));
        } else {
            return _run(query_vecs.get_all(), query_vecs.get_num_vecs(), hier_graph, false, {});
        }
    }

    /** query(query_vec, graph): at most topk entries (hierarchical_graph_router.hpp:164-174). */
    template <bool RandomSeeding = false, bool enable_early_stop = false, typename HierarchicalGraphT>
    auto query(const vec_ele_t* query_vec, const HierarchicalGraphT& hier_graph) const -> knn_results_t {
        static_assert(!RandomSeeding, "see batch_query");
        if constexpr (enable_early_stop) {
            static_assert(requires { hier_graph.rgraph_config(); hier_graph.pruning_config(); },
                          "Early stopping on a bare graph requires explicit rgraph and pruning configs");
            return query<RandomSeeding, true>(query_vec, hier_graph, hier_graph.rgraph_config(),
                                              hier_graph.pruning_config());
        } else {
            return _trim(_run(query_vec, 1, hier_graph, false, {}));
        }
    }

    /** query with explicit configurations (hierarchical_graph_router.hpp:176-190). */
    template <bool RandomSeeding = false, bool enable_early_stop = false, typename HierarchicalGraphT,
              typename RGraphConfigT, typename PruningConfigT>
    auto query(const vec_ele_t* query_vec, const HierarchicalGraphT& hier_graph, const RGraphConfigT& rgraph_config,
               const PruningConfigT& pruning_config) const -> knn_results_t {
        static_assert(!RandomSeeding, "see batch_query");
        if constexpr (enable_early_stop) {
            return _trim(_run(query_vec, 1, hier_graph, false,
                              _config_thresholds(hier_graph, rgraph_config, pruning_config)));
        } else {
            return _trim(_run(query_vec, 1, hier_graph, false, {}));
        }
    }

    /** batch_query_l0_only (hierarchical_graph_router.hpp:353-385). */
    template <bool RandomSeeding = false, typename HierarchicalGraphT>
    auto batch_query_l0_only(const query_vecs_t& query_vecs, const HierarchicalGraphT& hier_graph) const
        -> knn_results_t {
        static_assert(!RandomSeeding, "see batch_query");
        static_assert(HierarchicalGraphT::is_compacted, "batch_query_l0_only is only defined for compact graphs.");
        return _run(query_vecs.get_all(), query_vecs.get_num_vecs(), hier_graph, true, {});
    }

private:
    struct Device {
        std::mutex mu;   // early-stop setting + launch of one call
        uint64_t fingerprint = 0;
        artea_gpu_index* index = nullptr;
        artea_gpu_router* router = nullptr;
        ~Device() {
            if (router) artea_gpu_router_destroy(router);
            if (index) artea_gpu_index_destroy(index);
        }
    };
    struct State {
        std::mutex mu;
        std::map<const void*, std::shared_ptr<Device>> by_graph;
    };

    // Sizes, storage addresses and about 6,000 sampled words of the graph
    // (splitmix64 steps): a different graph at the same address differs here.
    template <typename HierarchicalGraphT>
    static auto _fingerprint(const HierarchicalGraphT& g) -> uint64_t {
        uint64_t h = 0x9E3779B97F4A7C15ull;
        auto mix = [&h](uint64_t x) {
            h ^= x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
            h ^= h >> 30;
            h *= 0xBF58476D1CE4E5B9ull;
            h ^= h >> 27;
        };
        const uint32_t n = g.get_num_vertices();
        const auto top = g.top_occupied_level_id();
        const auto ids = g.neighbor_ids();
        mix(n);
        mix(static_cast<uint64_t>(top));
        mix(g.entry_point_vid());
        mix(ids.size());
        mix(reinterpret_cast<uintptr_t>(ids.data()));
        for (std::size_t i = 0, step = std::max<std::size_t>(ids.size() / 4096, 1); i < ids.size(); i += step)
            mix(ids[i]);
        for (uint32_t v = 0, step = std::max<uint32_t>(n / 1024, 1); v < n; v += step) {
            const auto& info = g.get_vertex_info(v);
            mix((static_cast<uint64_t>(info.highest_level) << 32) | info.local_vid);
        }
        if (top != HierarchicalGraphT::invalid_level_id) {
            for (uint32_t lvl = 0; lvl <= static_cast<uint32_t>(top); ++lvl) {
                const auto off = g.get_nbr_offsets(lvl);
                mix(reinterpret_cast<uintptr_t>(off.data()));
                mix(off.size());
                if (!off.empty()) mix(off.back());
            }
        }
        return h;
    }

    template <typename HierarchicalGraphT>
    auto _device_for(const HierarchicalGraphT& g) const -> std::shared_ptr<Device> {
        const uint64_t fp = _fingerprint(g);
        std::lock_guard<std::mutex> lk(_state->mu);
        auto it = _state->by_graph.find(&g);
        if (it != _state->by_graph.end()) {
            if (it->second->fingerprint == fp) return it->second;
            _state->by_graph.erase(it);   // another graph now lives at this address
        }
        // compact::HierarchicalGraph -> artea_gpu_graph_desc
        // (compact_structure/hierarchical_graph.hpp:46-49, 83-121).
        const uint32_t n = g.get_num_vertices();
        const uint32_t top = g.top_occupied_level_id();
        const bool empty = top == HierarchicalGraphT::invalid_level_id;
        std::vector<const uint64_t*> offsets;
        std::vector<uint64_t> sizes;
        if (!empty) {
            for (uint32_t h = 0; h <= top; ++h) {
                offsets.push_back(g.get_nbr_offsets(h).data());
                sizes.push_back(g.get_vids_with_highest_level(h).size());
            }
        } else {
            sizes.push_back(0);
        }
        static_assert(sizeof(typename HierarchicalGraphT::VertexInfo) == 8, "vertex table of {level, local id}");
        artea_gpu_graph_desc d{};
        d.num_vertices = n;
        d.top_level = empty ? 0xFFFFFFFFu : top;
        d.ul_max_nbr_size = g.ul_max_nbr_size();
        d.bl_max_nbr_size = g.bl_max_nbr_size();
        d.entry_point_vid = g.entry_point_vid();
        d.vertex_info = n ? reinterpret_cast<const uint32_t*>(&g.get_vertex_info(0)) : nullptr;
        d.group_offsets = offsets.data();
        d.group_sizes = sizes.data();
        d.neighbor_ids = g.neighbor_ids().data();
        d.num_neighbor_ids = g.neighbor_ids().size();
        auto dev = std::make_shared<Device>();
        dev->fingerprint = fp;
        detail::check(artea_gpu_index_create(&d, _vecs.get_all(), _vecs.get_num_vecs(), _vecs.get_vec_dim(),
                                             _opts.device, &dev->index),
                      "artea_gpu_index_create");
        artea_gpu_router_opts o{};
        o.metric = detail::metric_code<RouterTraitsT>();
        o.mode = _opts.mode;
        o.schedule = _opts.schedule;
        detail::check(artea_gpu_router_create(dev->index, _topk, _queue, &o, &dev->router), "artea_gpu_router_create");
        _state->by_graph.emplace(&g, dev);
        return dev;
    }

    // Per-level configuration thresholds, index = level, for levels 1..top of
    // g (empty when g has no level above 0: none is needed, :392-393).
    template <typename HierarchicalGraphT, typename RGraphConfigT, typename PruningConfigT>
    static auto _config_thresholds(const HierarchicalGraphT& g, const RGraphConfigT& rgraph_config,
                                   const PruningConfigT& pruning_config) -> std::vector<float> {
        const auto top = g.top_occupied_level_id();
        if (top == HierarchicalGraphT::invalid_level_id || top == 0) return {};
        std::vector<float> thr(static_cast<std::size_t>(top) + 1, 0.0f);
        for (uint32_t h = 1; h <= static_cast<uint32_t>(top); ++h)
            thr[h] = static_cast<float>(rgraph_config.early_stop_threshold(h, pruning_config));
        return thr;
    }

    static auto _trim(knn_results_t res) -> knn_results_t {
        while (!res.empty() && res.back().is_invalid()) res.pop_back();
        return res;
    }

    template <typename HierarchicalGraphT>
    auto _run(const vec_ele_t* queries, uint32_t nq, const HierarchicalGraphT& g, bool l0_only,
              const std::vector<float>& early_stop) const -> knn_results_t {
        const std::shared_ptr<Device> held = _device_for(g);   // kept alive for this call
        Device& dev = *held;
        std::lock_guard<std::mutex> lk(dev.mu);
        const int es = early_stop.empty()
                           ? artea_gpu_router_set_early_stop(dev.router, nullptr, 0)
                           : artea_gpu_router_set_early_stop(dev.router, early_stop.data(),
                                                             static_cast<uint32_t>(early_stop.size()));
        if (es != ARTEA_GPU_OK && std::string(artea_gpu_last_error()).find("not representable") != std::string::npos)
            throw std::overflow_error(artea_gpu_last_error());
        detail::check(es, "artea_gpu_router_set_early_stop");
        knn_results_t results(static_cast<std::size_t>(nq) * _topk, candidate_entry_t::make_invalid_entry());
        if (nq == 0 || _topk == 0) return results;
        std::vector<uint64_t> words(static_cast<std::size_t>(nq) * _topk);
        const int rc = l0_only
                           ? artea_gpu_batch_query_l0_only(dev.router, queries, nq, _topk, words.data(), nullptr)
                           : artea_gpu_batch_query(dev.router, queries, nq, nullptr, nullptr, _topk, words.data(),
                                                   nullptr);
        detail::check(rc, "artea_gpu_batch_query");
        std::memcpy(static_cast<void*>(results.data()), words.data(), words.size() * sizeof(uint64_t));
        return results;
    }

    const vector_array_t& _vecs;
    const dist_func_t& _dist;
    uint32_t _topk;
    vertex_num_t _queue;
    RouterOptions _opts;
    std::shared_ptr<State> _state;
};

}  // namespace cuda
}  // namespace artea
