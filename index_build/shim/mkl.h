// Stand-in for the three MKL VSL calls ARTEA uses (vslNewStream, viRngUniform,
// vslDeleteStream). MKL is not installed in this image. Streams are
// std::mt19937 engines; viRngUniform draws integers uniformly in [a, b).
// These draws only steer index construction (insertion shuffle, L0 random
// prefill) and the optional random seeding of queries, never the default
// query path, so a built graph differs from an MKL-built one only in which
// random choices were made.
#pragma once
#include <cstdint>
#include <random>

typedef int MKL_INT;
typedef void* VSLStreamStatePtr;

#define VSL_BRNG_MT19937 0x00200000
#define VSL_RNG_METHOD_UNIFORM_STD 0
#define VSL_STATUS_OK 0

inline int vslNewStream(VSLStreamStatePtr* stream, MKL_INT /*brng*/, unsigned int seed) {
    *stream = new std::mt19937(seed);
    return VSL_STATUS_OK;
}

inline int vslDeleteStream(VSLStreamStatePtr* stream) {
    delete static_cast<std::mt19937*>(*stream);
    *stream = nullptr;
    return VSL_STATUS_OK;
}

inline int viRngUniform(MKL_INT /*method*/, VSLStreamStatePtr stream, MKL_INT n, int* r, int a, int b) {
    auto& eng = *static_cast<std::mt19937*>(stream);
    if (b <= a) {
        for (MKL_INT i = 0; i < n; ++i) r[i] = a;
        return VSL_STATUS_OK;
    }
    std::uniform_int_distribution<std::int64_t> dist(a, static_cast<std::int64_t>(b) - 1);
    for (MKL_INT i = 0; i < n; ++i) r[i] = static_cast<int>(dist(eng));
    return VSL_STATUS_OK;
}
