// Minimal stand-in for the part of oneTBB that the ARTEA headers use.
//
// oneTBB is not installed in this image and there is no network, so the ARTEA
// builder and router headers are compiled against this shim. It provides one
// process-wide pool of worker threads that hands out range chunks through an
// atomic counter (dynamic scheduling, caller thread participates). Nested
// parallel calls issued from inside a running parallel region execute inline on
// the calling thread, which keeps nesting deadlock-free.
//
// Thread count: ARTEA_SHIM_THREADS if set, else std::thread::hardware_concurrency().
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdlib>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace tbb {
namespace shim {

inline thread_local bool tls_in_parallel = false;

class pool {
public:
    static pool& get() {
        static pool instance;
        return instance;
    }

    /// Threads that take part in a parallel region (workers + caller), after any global limit.
    int concurrency() const {
        const int lim = _limit.load(std::memory_order_relaxed);
        const int all = static_cast<int>(_workers.size()) + 1;
        return lim > 0 ? std::min(lim, all) : all;
    }

    void set_limit(int lim) { _limit.store(lim, std::memory_order_relaxed); }
    int limit() const { return _limit.load(std::memory_order_relaxed); }

    /// Run fn(chunk) for chunk in [0, nchunks) over the pool; returns when all are done.
    void run(std::size_t nchunks, const std::function<void(std::size_t)>& fn) {
        if (nchunks == 0) return;
        if (tls_in_parallel || concurrency() <= 1 || nchunks == 1) {
            const bool outer = tls_in_parallel;
            tls_in_parallel = true;
            try {
                for (std::size_t c = 0; c < nchunks; ++c) fn(c);
            } catch (...) {
                tls_in_parallel = outer;
                throw;
            }
            tls_in_parallel = outer;
            return;
        }
        std::lock_guard<std::mutex> serial(_job_serial);
        {
            std::lock_guard<std::mutex> lk(_mu);
            _fn = &fn;
            _nchunks = nchunks;
            _next.store(0, std::memory_order_relaxed);
            _done.store(0, std::memory_order_relaxed);
            _error = nullptr;
            _active_workers = std::min<int>(concurrency() - 1, static_cast<int>(_workers.size()));
            _busy = 0;
            ++_generation;
        }
        _cv.notify_all();
        work_loop();
        {
            std::unique_lock<std::mutex> lk(_mu);
            _cv_done.wait(lk, [&] { return _done.load() == _nchunks && _busy == 0; });
            _fn = nullptr;
        }
        if (_error) std::rethrow_exception(_error);
    }

private:
    pool() {
        int n = 0;
        if (const char* env = std::getenv("ARTEA_SHIM_THREADS")) n = std::atoi(env);
        if (n <= 0) n = static_cast<int>(std::thread::hardware_concurrency());
        if (n <= 0) n = 1;
        for (int i = 0; i < n - 1; ++i) {
            _workers.emplace_back([this, i] { worker_main(i); });
        }
    }

    ~pool() {
        {
            std::lock_guard<std::mutex> lk(_mu);
            _stop = true;
            ++_generation;
        }
        _cv.notify_all();
        for (auto& t : _workers) t.join();
    }

    void work_loop() {
        const bool outer = tls_in_parallel;
        tls_in_parallel = true;
        for (;;) {
            const std::size_t c = _next.fetch_add(1, std::memory_order_relaxed);
            if (c >= _nchunks) break;
            try {
                (*_fn)(c);
            } catch (...) {
                std::lock_guard<std::mutex> lk(_mu);
                if (!_error) _error = std::current_exception();
            }
            if (_done.fetch_add(1, std::memory_order_acq_rel) + 1 == _nchunks) {
                std::lock_guard<std::mutex> lk(_mu);
                _cv_done.notify_all();
            }
        }
        tls_in_parallel = outer;
    }

    void worker_main(int index) {
        std::size_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(_mu);
                _cv.wait(lk, [&] { return _stop || _generation != seen; });
                if (_stop) return;
                seen = _generation;
                if (index >= _active_workers || _fn == nullptr) continue;
                ++_busy;
            }
            work_loop();
            {
                std::lock_guard<std::mutex> lk(_mu);
                --_busy;
                _cv_done.notify_all();
            }
        }
    }

    std::vector<std::thread> _workers;
    std::mutex _mu;
    std::mutex _job_serial;
    std::condition_variable _cv;
    std::condition_variable _cv_done;
    const std::function<void(std::size_t)>* _fn = nullptr;
    std::size_t _nchunks = 0;
    std::atomic<std::size_t> _next{0};
    std::atomic<std::size_t> _done{0};
    std::exception_ptr _error;
    int _active_workers = 0;
    int _busy = 0;
    std::size_t _generation = 0;
    bool _stop = false;
    std::atomic<int> _limit{0};
};

}  // namespace shim
}  // namespace tbb
