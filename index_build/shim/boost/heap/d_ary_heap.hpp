// Declaration-only stand-in for boost::heap::d_ary_heap. Boost is not in this
// image; the ARTEA header that names this type (the boost-backed candidate
// queue) is never instantiated by the index builder or the query oracle.
#pragma once

namespace boost {
namespace heap {
template <unsigned Arity> struct arity {};
template <typename Compare> struct compare {};
template <typename T, typename... Options> class d_ary_heap;
}  // namespace heap
}  // namespace boost
