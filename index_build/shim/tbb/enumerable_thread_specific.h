// Shim of tbb::enumerable_thread_specific: one lazily constructed T per thread,
// stable addresses, iteration over all constructed copies.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <iterator>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace tbb {
namespace shim {

inline std::uint64_t next_ets_id() {
    static std::atomic<std::uint64_t> counter{1};
    return counter.fetch_add(1, std::memory_order_relaxed);
}

/// Per-thread cache of the most recently used (instance id -> element) lookups.
struct ets_cache {
    static constexpr int kSlots = 16;
    std::uint64_t ids[kSlots] = {};
    void* ptrs[kSlots] = {};
    int next = 0;
};
inline thread_local ets_cache tls_ets_cache;

}  // namespace shim

template <typename T>
class enumerable_thread_specific {
    struct slot {
        std::thread::id owner;
        std::unique_ptr<T> value;
    };

public:
    using value_type = T;
    using reference = T&;
    using const_reference = const T&;
    using size_type = std::size_t;

    template <typename Base, typename Ref>
    class basic_iterator {
    public:
        using iterator_category = std::random_access_iterator_tag;
        using value_type = T;
        using difference_type = std::ptrdiff_t;
        using pointer = std::remove_reference_t<Ref>*;
        using reference = Ref;
        basic_iterator() = default;
        basic_iterator(Base it) : _it(it) {}
        Ref operator*() const { return *(_it->value); }
        pointer operator->() const { return _it->value.get(); }
        basic_iterator& operator++() { ++_it; return *this; }
        basic_iterator operator++(int) { auto t = *this; ++_it; return t; }
        bool operator==(const basic_iterator& o) const { return _it == o._it; }
        bool operator!=(const basic_iterator& o) const { return _it != o._it; }
    private:
        Base _it{};
    };
    using iterator = basic_iterator<typename std::vector<slot>::iterator, T&>;
    using const_iterator = basic_iterator<typename std::vector<slot>::const_iterator, const T&>;

    enumerable_thread_specific() : _make([] { return std::make_unique<T>(); }) {}

    template <typename Arg,
              typename = std::enable_if_t<!std::is_same_v<std::decay_t<Arg>, enumerable_thread_specific>>>
    explicit enumerable_thread_specific(Arg&& arg) {
        if constexpr (std::is_invocable_v<std::decay_t<Arg>&>) {
            auto f = std::forward<Arg>(arg);
            _make = [f]() mutable { return std::make_unique<T>(f()); };
        } else {
            T exemplar(std::forward<Arg>(arg));
            _make = [exemplar]() { return std::make_unique<T>(exemplar); };
        }
    }

    enumerable_thread_specific(const enumerable_thread_specific&) = delete;
    enumerable_thread_specific& operator=(const enumerable_thread_specific&) = delete;
    enumerable_thread_specific(enumerable_thread_specific&& o) noexcept
        : _make(std::move(o._make)), _slots(std::move(o._slots)) {
        o._id = shim::next_ets_id();
    }
    enumerable_thread_specific& operator=(enumerable_thread_specific&& o) noexcept {
        if (this != &o) {
            std::lock_guard<std::mutex> lk(_mu);
            _make = std::move(o._make);
            _slots = std::move(o._slots);
            _id = shim::next_ets_id();
        }
        return *this;
    }

    T& local() {
        bool exists;
        return local(exists);
    }

    T& local(bool& exists) {
        auto& cache = shim::tls_ets_cache;
        for (int i = 0; i < shim::ets_cache::kSlots; ++i) {
            if (cache.ids[i] == _id) {
                exists = true;
                return *static_cast<T*>(cache.ptrs[i]);
            }
        }
        T* found = nullptr;
        {
            std::lock_guard<std::mutex> lk(_mu);
            const auto me = std::this_thread::get_id();
            for (auto& s : _slots) {
                if (s.owner == me) { found = s.value.get(); break; }
            }
            exists = found != nullptr;
            if (!found) {
                _slots.push_back(slot{me, _make()});
                found = _slots.back().value.get();
            }
        }
        cache.ids[cache.next] = _id;
        cache.ptrs[cache.next] = found;
        cache.next = (cache.next + 1) % shim::ets_cache::kSlots;
        return *found;
    }

    size_type size() const { return _slots.size(); }
    bool empty() const { return _slots.empty(); }
    void clear() {
        std::lock_guard<std::mutex> lk(_mu);
        _slots.clear();
        _id = shim::next_ets_id();
    }

    iterator begin() { return iterator(_slots.begin()); }
    iterator end() { return iterator(_slots.end()); }
    const_iterator begin() const { return const_iterator(_slots.cbegin()); }
    const_iterator end() const { return const_iterator(_slots.cend()); }

    template <typename F>
    void combine_each(F f) {
        for (auto& s : _slots) f(*s.value);
    }
    template <typename F>
    T combine(F f) {
        if (_slots.empty()) return *_make();
        T acc = *_slots.front().value;
        for (std::size_t i = 1; i < _slots.size(); ++i) acc = f(acc, *_slots[i].value);
        return acc;
    }

private:
    std::function<std::unique_ptr<T>()> _make;
    std::vector<slot> _slots;
    std::mutex _mu;
    std::uint64_t _id = shim::next_ets_id();
};

}  // namespace tbb
