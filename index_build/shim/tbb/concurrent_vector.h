// Shim of tbb::concurrent_vector: append-only growth from many threads with
// stable element addresses. Storage is a table of geometrically growing
// segments; appends take a mutex, construct the element, then publish the new
// size, so a reader that sees size() = n can read elements [0, n).
#pragma once
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <iterator>
#include <memory>
#include <mutex>
#include <new>
#include <type_traits>
#include <utility>

namespace tbb {

template <typename T>
class concurrent_vector {
    static constexpr std::size_t kBase = 16;       // size of segment 0
    static constexpr std::size_t kMaxSegments = 48;

    static std::size_t segment_of(std::size_t i) {
        std::size_t q = i / kBase + 1;
        std::size_t s = 0;
        while (q >>= 1) ++s;
        return s;
    }
    static std::size_t segment_start(std::size_t s) { return kBase * ((std::size_t(1) << s) - 1); }
    static std::size_t segment_size(std::size_t s) { return kBase << s; }

public:
    using value_type = T;
    using size_type = std::size_t;
    using difference_type = std::ptrdiff_t;
    using reference = T&;
    using const_reference = const T&;

    template <typename Owner, typename Ref>
    class basic_iterator {
    public:
        using iterator_concept = std::random_access_iterator_tag;
        using iterator_category = std::random_access_iterator_tag;
        using value_type = T;
        using difference_type = std::ptrdiff_t;
        using pointer = std::remove_reference_t<Ref>*;
        using reference = Ref;

        basic_iterator() = default;
        basic_iterator(Owner* v, std::size_t i) : _v(v), _i(i) {}
        template <typename O2, typename R2,
                  typename = std::enable_if_t<std::is_convertible_v<O2*, Owner*>>>
        basic_iterator(const basic_iterator<O2, R2>& o) : _v(o._v), _i(o._i) {}

        Ref operator*() const { return (*_v)[_i]; }
        pointer operator->() const { return &(*_v)[_i]; }
        Ref operator[](difference_type n) const { return (*_v)[_i + n]; }
        basic_iterator& operator++() { ++_i; return *this; }
        basic_iterator operator++(int) { auto t = *this; ++_i; return t; }
        basic_iterator& operator--() { --_i; return *this; }
        basic_iterator operator--(int) { auto t = *this; --_i; return t; }
        basic_iterator& operator+=(difference_type n) { _i += n; return *this; }
        basic_iterator& operator-=(difference_type n) { _i -= n; return *this; }
        friend basic_iterator operator+(basic_iterator a, difference_type n) { a += n; return a; }
        friend basic_iterator operator+(difference_type n, basic_iterator a) { a += n; return a; }
        friend basic_iterator operator-(basic_iterator a, difference_type n) { a -= n; return a; }
        friend difference_type operator-(const basic_iterator& a, const basic_iterator& b) {
            return static_cast<difference_type>(a._i) - static_cast<difference_type>(b._i);
        }
        friend bool operator==(const basic_iterator& a, const basic_iterator& b) { return a._i == b._i; }
        friend auto operator<=>(const basic_iterator& a, const basic_iterator& b) { return a._i <=> b._i; }

        Owner* _v = nullptr;
        std::size_t _i = 0;
    };
    using iterator = basic_iterator<concurrent_vector, T&>;
    using const_iterator = basic_iterator<const concurrent_vector, const T&>;

    concurrent_vector() = default;
    explicit concurrent_vector(size_type n) { grow_to_at_least(n); }
    concurrent_vector(const concurrent_vector& o) {
        for (size_type i = 0; i < o.size(); ++i) push_back(o[i]);
    }
    concurrent_vector(concurrent_vector&& o) noexcept {
        for (std::size_t s = 0; s < kMaxSegments; ++s) {
            _segments[s].store(o._segments[s].load());
            o._segments[s].store(nullptr);
        }
        _size.store(o._size.load());
        o._size.store(0);
    }
    concurrent_vector& operator=(const concurrent_vector& o) {
        if (this != &o) {
            clear();
            for (size_type i = 0; i < o.size(); ++i) push_back(o[i]);
        }
        return *this;
    }
    concurrent_vector& operator=(concurrent_vector&& o) noexcept {
        if (this != &o) {
            destroy_all();
            for (std::size_t s = 0; s < kMaxSegments; ++s) {
                _segments[s].store(o._segments[s].load());
                o._segments[s].store(nullptr);
            }
            _size.store(o._size.load());
            o._size.store(0);
        }
        return *this;
    }
    ~concurrent_vector() { destroy_all(); }

    size_type size() const { return _size.load(std::memory_order_acquire); }
    bool empty() const { return size() == 0; }
    size_type capacity() const {
        size_type c = 0;
        for (std::size_t s = 0; s < kMaxSegments; ++s)
            if (_segments[s].load(std::memory_order_acquire)) c = segment_start(s) + segment_size(s);
        return c;
    }

    T& operator[](size_type i) { return *slot(i); }
    const T& operator[](size_type i) const { return *slot(i); }
    T& at(size_type i) { return *slot(i); }
    const T& at(size_type i) const { return *slot(i); }
    T& front() { return *slot(0); }
    T& back() { return *slot(size() - 1); }
    const T& front() const { return *slot(0); }
    const T& back() const { return *slot(size() - 1); }

    iterator push_back(const T& v) { return emplace_back(v); }
    iterator push_back(T&& v) { return emplace_back(std::move(v)); }

    template <typename... Args>
    iterator emplace_back(Args&&... args) {
        std::lock_guard<std::mutex> lk(_mu);
        const size_type i = _size.load(std::memory_order_relaxed);
        T* p = raw_slot_alloc(i);
        ::new (static_cast<void*>(p)) T(std::forward<Args>(args)...);
        _size.store(i + 1, std::memory_order_release);
        return iterator(this, i);
    }

    iterator grow_by(size_type n) {
        std::lock_guard<std::mutex> lk(_mu);
        const size_type i0 = _size.load(std::memory_order_relaxed);
        for (size_type k = 0; k < n; ++k) ::new (static_cast<void*>(raw_slot_alloc(i0 + k))) T();
        _size.store(i0 + n, std::memory_order_release);
        return iterator(this, i0);
    }

    iterator grow_to_at_least(size_type n) {
        std::lock_guard<std::mutex> lk(_mu);
        const size_type i0 = _size.load(std::memory_order_relaxed);
        for (size_type k = i0; k < n; ++k) ::new (static_cast<void*>(raw_slot_alloc(k))) T();
        if (n > i0) _size.store(n, std::memory_order_release);
        return iterator(this, std::min(i0, n));
    }

    void reserve(size_type n) {
        std::lock_guard<std::mutex> lk(_mu);
        if (n) raw_slot_alloc(n - 1);
    }

    void clear() {
        const size_type n = size();
        for (size_type i = 0; i < n; ++i) slot(i)->~T();
        _size.store(0, std::memory_order_release);
    }

    iterator begin() { return iterator(this, 0); }
    iterator end() { return iterator(this, size()); }
    const_iterator begin() const { return const_iterator(this, 0); }
    const_iterator end() const { return const_iterator(this, size()); }
    const_iterator cbegin() const { return const_iterator(this, 0); }
    const_iterator cend() const { return const_iterator(this, size()); }

private:
    T* slot(size_type i) const {
        const std::size_t s = segment_of(i);
        T* seg = _segments[s].load(std::memory_order_acquire);
        return seg + (i - segment_start(s));
    }

    T* raw_slot_alloc(size_type i) {
        const std::size_t s_last = segment_of(i);
        for (std::size_t s = 0; s <= s_last; ++s) {
            if (!_segments[s].load(std::memory_order_relaxed)) {
                void* mem = ::operator new(segment_size(s) * sizeof(T), std::align_val_t(alignof(T) < 64 ? 64 : alignof(T)));
                _segments[s].store(static_cast<T*>(mem), std::memory_order_release);
            }
        }
        return slot(i);
    }

    void destroy_all() {
        clear();
        for (std::size_t s = 0; s < kMaxSegments; ++s) {
            if (T* seg = _segments[s].load()) {
                ::operator delete(static_cast<void*>(seg), std::align_val_t(alignof(T) < 64 ? 64 : alignof(T)));
                _segments[s].store(nullptr);
            }
        }
    }

    std::atomic<T*> _segments[kMaxSegments] = {};
    std::atomic<size_type> _size{0};
    std::mutex _mu;
};

}  // namespace tbb
