// Shim of tbb::parallel_reduce (functional form) over the shared worker pool.
// Chunk partial results are joined left to right in chunk order.
#pragma once
#include <cstddef>
#include <vector>
#include <tbb/parallel_for.h>

namespace tbb {

template <typename Value, typename T, typename RealBody, typename Reduction>
T parallel_reduce(const blocked_range<Value>& range, const T& identity, const RealBody& body,
                  const Reduction& reduction) {
    const std::size_t chunks = shim::chunk_count(range.size(), range.grainsize());
    if (chunks == 0) return identity;
    std::vector<T> partial(chunks, identity);
    shim::pool::get().run(chunks, [&](std::size_t c) {
        partial[c] = body(shim::chunk_of(range, chunks, c), identity);
    });
    T acc = partial[0];
    for (std::size_t c = 1; c < chunks; ++c) acc = reduction(acc, partial[c]);
    return acc;
}

}  // namespace tbb
