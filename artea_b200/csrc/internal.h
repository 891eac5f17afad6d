// Host-side internals shared by the C-ABI translation units: the index
// structure, error macro, device guard and device allocation helpers.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/artea_gpu.h"
#include "common.h"
#include "search.cuh"

using artea_gpu::fail;

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t _e = (expr);                                                                    \
        if (_e != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// A device-resident graph plus its vectors (artea_gpu_index_create).
struct artea_gpu_index {
    int device = 0;
    uint32_t n = 0, dim = 0, top = artea_gpu::kInvalidLevel, entry = 0, ul = 0, bl = 0;
    uint32_t l0_unique = 0;   // level-0 rows of <= 64 ids hold distinct ids (checked at upload)
    uint32_t nvecs = 0;       // vector rows uploaded (brute force scans all of them)
    float* d_vecs = nullptr;
    float* d_xsq = nullptr;   // squared norm of every vector row (the cosine distance's x.x)
    uint2* d_vinfo = nullptr;
    uint32_t* d_nbrs = nullptr;
    uint64_t* d_offsets = nullptr;
    unsigned long long* d_l0row = nullptr;
    const uint64_t* group_ptr[artea_gpu::kMaxGroups] = {};
    uint64_t n_offsets = 0;   // entries of d_offsets (all groups, with their end sentinels)
    uint64_t n_nbrs = 0;      // entries of d_nbrs in use
    uint64_t bytes = 0;
};

namespace artea_gpu {

// Makes a device current for a scope.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

template <typename T>
inline int dev_alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return ARTEA_GPU_OK;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? ARTEA_GPU_ENOMEM : ARTEA_GPU_ECUDA,
                    std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return ARTEA_GPU_OK;
}

template <typename T>
inline void dev_free(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// Steps of index creation shared by the host-graph and the snapshot paths
// (artea_gpu.cu).
// Checks dim / vector count / device and uploads the vectors into a new index.
int index_begin(uint32_t num_vertices, const float* vectors, uint32_t num_vectors, uint32_t dim, int device,
                artea_gpu_index** out);
// With d_vinfo, d_nbrs and d_offsets in place (group h's offsets at
// group_offsets_host[h] on the host): the level-0 row descriptors and the
// row-repeat check.
int index_finish_l0(artea_gpu_index* ix, const uint32_t* vertex_info, const uint64_t* const* group_offsets_host);

}  // namespace artea_gpu
