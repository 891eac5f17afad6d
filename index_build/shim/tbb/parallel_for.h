// Shim of tbb::parallel_for over the shared worker pool (see detail_pool.h).
#pragma once
#include <algorithm>
#include <cstddef>
#include <tbb/blocked_range.h>
#include <tbb/detail_pool.h>

namespace tbb {
namespace shim {

/// Number of chunks a range of `n` items with the given grain size is cut into.
inline std::size_t chunk_count(std::size_t n, std::size_t grain) {
    if (n == 0) return 0;
    const std::size_t target = static_cast<std::size_t>(pool::get().concurrency()) * 16;
    std::size_t chunks = std::min(n, target);
    if (grain > 1) chunks = std::max<std::size_t>(std::min(chunks, (n + grain - 1) / grain), 1);
    return chunks;
}

template <typename Value>
blocked_range<Value> chunk_of(const blocked_range<Value>& r, std::size_t chunks, std::size_t c) {
    const std::size_t n = r.size();
    const std::size_t lo = n * c / chunks;
    const std::size_t hi = n * (c + 1) / chunks;
    return blocked_range<Value>(static_cast<Value>(r.begin() + lo), static_cast<Value>(r.begin() + hi),
                                r.grainsize());
}

}  // namespace shim

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body) {
    const std::size_t chunks = shim::chunk_count(range.size(), range.grainsize());
    if (chunks == 0) return;
    shim::pool::get().run(chunks, [&](std::size_t c) { body(shim::chunk_of(range, chunks, c)); });
}

template <typename Value, typename Body, typename Partitioner>
void parallel_for(const blocked_range<Value>& range, const Body& body, Partitioner&) {
    parallel_for(range, body);
}

template <typename Index, typename Function>
void parallel_for(Index first, Index last, const Function& f) {
    if (!(first < last)) return;
    parallel_for(blocked_range<Index>(first, last), [&](const blocked_range<Index>& r) {
        for (Index i = r.begin(); i < r.end(); ++i) f(i);
    });
}

template <typename Index, typename Function>
void parallel_for(Index first, Index last, Index step, const Function& f) {
    if (!(first < last) || step <= 0) return;
    const Index count = (last - first + step - 1) / step;
    parallel_for(blocked_range<Index>(0, count), [&](const blocked_range<Index>& r) {
        for (Index i = r.begin(); i < r.end(); ++i) f(first + i * step);
    });
}

}  // namespace tbb
