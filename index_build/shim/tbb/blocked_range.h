// Shim of tbb::blocked_range (see detail_pool.h for why the shim exists).
#pragma once
#include <cstddef>

namespace tbb {

struct split {};

template <typename Value>
class blocked_range {
public:
    using const_iterator = Value;
    using size_type = std::size_t;

    blocked_range() = default;
    blocked_range(Value begin_, Value end_, size_type grainsize_ = 1)
        : _begin(begin_), _end(end_), _grainsize(grainsize_ ? grainsize_ : 1) {}

    const_iterator begin() const { return _begin; }
    const_iterator end() const { return _end; }
    size_type size() const { return _end > _begin ? size_type(_end - _begin) : 0; }
    size_type grainsize() const { return _grainsize; }
    bool empty() const { return !(_begin < _end); }
    bool is_divisible() const { return _grainsize < size(); }

private:
    Value _begin{};
    Value _end{};
    size_type _grainsize = 1;
};

}  // namespace tbb
