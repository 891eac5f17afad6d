// Shim of tbb::global_control (max_allowed_parallelism only).
#pragma once
#include <cstddef>
#include <tbb/detail_pool.h>

namespace tbb {

class global_control {
public:
    enum parameter { max_allowed_parallelism, thread_stack_size };
    global_control(parameter p, std::size_t value) : _param(p) {
        if (_param == max_allowed_parallelism) {
            _previous = shim::pool::get().limit();
            shim::pool::get().set_limit(static_cast<int>(value));
        }
    }
    ~global_control() {
        if (_param == max_allowed_parallelism) shim::pool::get().set_limit(_previous);
    }
    global_control(const global_control&) = delete;
    global_control& operator=(const global_control&) = delete;

private:
    parameter _param;
    int _previous = 0;
};

}  // namespace tbb
