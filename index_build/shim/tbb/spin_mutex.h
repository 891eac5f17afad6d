// Shim of tbb::spin_mutex (test-and-test-and-set lock with yield).
#pragma once
#include <atomic>
#include <thread>

namespace tbb {

class spin_mutex {
public:
    spin_mutex() = default;
    spin_mutex(const spin_mutex&) = delete;
    spin_mutex& operator=(const spin_mutex&) = delete;

    void lock() {
        for (;;) {
            if (!_flag.exchange(true, std::memory_order_acquire)) return;
            while (_flag.load(std::memory_order_relaxed)) std::this_thread::yield();
        }
    }
    bool try_lock() { return !_flag.exchange(true, std::memory_order_acquire); }
    void unlock() { _flag.store(false, std::memory_order_release); }

    class scoped_lock {
    public:
        scoped_lock() = default;
        explicit scoped_lock(spin_mutex& m) { acquire(m); }
        ~scoped_lock() { release(); }
        void acquire(spin_mutex& m) { _m = &m; m.lock(); }
        bool try_acquire(spin_mutex& m) {
            if (m.try_lock()) { _m = &m; return true; }
            return false;
        }
        void release() {
            if (_m) { _m->unlock(); _m = nullptr; }
        }

    private:
        spin_mutex* _m = nullptr;
    };

private:
    std::atomic<bool> _flag{false};
};

}  // namespace tbb
