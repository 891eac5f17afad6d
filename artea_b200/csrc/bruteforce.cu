// Exact brute-force k-NN on the GPU: BruteforceRouter::query / batch_query and
// the subset overloads (router/bruteforce_router.hpp:74-160, 100-125, 164-190).
// This is the step after the query path (recall@k needs ground truth); the
// distances are the reference's, bit for bit: one thread evaluates a whole row,
// holding the 16 AVX-512 lane chains of utils/simd_distance.hpp:100-115 as
// eight packed FP32 pairs, then folds them with the _mm512_reduce_add_ps tree.
//
// Layout: a CTA takes kBfQueries queries (staged in shared memory) against a
// segment of the candidate rows; each thread loads one row chunk (16 floats)
// at a time and applies it to all the CTA's queries, so a row crosses HBM/L2
// once per CTA. Per query the CTA keeps a shared-memory list of (distance, vid)
// keys below the current k-th best; when a list fills, one warp sorts it and
// trims it to k. Several segments per query tile are merged by a second kernel.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/artea_gpu.h"
#include "common.h"
#include "internal.h"

namespace artea_gpu {
namespace {

constexpr int kBfQueries = 8;        // queries per CTA
constexpr int kBfThreads = 128;      // rows per round (one per thread)
constexpr uint32_t kBfMaxTopk = 1024;
constexpr uint64_t kMaxKey = ~0ull;
// CandidateEntry() (router/data_structures/candidate_entry.hpp:72-74): vid =
// invalid_vertex_id (all ones), distance 0 -- the padding of batch rows whose
// query has fewer than topk candidates (bruteforce_router.hpp:142, 177).
constexpr uint64_t kDefaultEntryWord = 0x00000000FFFFFFFFull;

// (distance, vid) as one unsigned key whose order is the order by distance,
// then vid (negative distances included: DOT).
__device__ __forceinline__ uint64_t order_key(float d, uint32_t vid) {
    uint32_t u = __float_as_uint(d);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return (static_cast<uint64_t>(u) << 32) | vid;
}
__device__ __forceinline__ uint64_t key_word(uint64_t key) {
    uint32_t u = static_cast<uint32_t>(key >> 32);
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return (static_cast<uint64_t>(u) << 32) | static_cast<uint32_t>(key);
}

// One sorted pass over n keys (n a power of two) by the calling warp.
__device__ void warp_bitonic_sort(uint64_t* a, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k2 = 2; k2 <= n; k2 <<= 1) {
        for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n; i += 32) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const uint64_t x = a[i], y = a[p];
                    const bool up = (i & k2) == 0;
                    if ((x > y) == up) {
                        a[i] = y;
                        a[p] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
}

__host__ __device__ inline uint32_t next_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Sort list q's first cnt keys (padding to a power of two) and keep the best k.
__device__ void trim_list(uint64_t* list, uint32_t cap, uint32_t* cnt, uint64_t* thr, uint32_t k) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = *cnt;
    const uint32_t p2 = next_pow2(max(n, 1u));
    for (uint32_t i = n + lane; i < p2; i += 32) list[i] = kMaxKey;
    __syncwarp();
    warp_bitonic_sort(list, p2);
    if (lane == 0) {
        const uint32_t kept = min(n, k);
        *cnt = kept;
        if (kept == k) *thr = list[k - 1];
    }
    __syncwarp();
    (void)cap;
}

struct BfArgs {
    const float* __restrict__ vecs;
    uint32_t dim;
    const uint32_t* __restrict__ subset;   // null: rows [0, n_rows)
    uint32_t n_rows;
    const float* __restrict__ queries;
    uint32_t nq;
    uint32_t k;
    uint32_t seg_len;                      // rows per segment (blockIdx.y)
    uint32_t segments;
    uint32_t list_cap;                     // power of two >= k + 2 * kBfThreads
    uint64_t* __restrict__ out;            // segments == 1: nq x k words
    uint64_t* __restrict__ part;           // segments > 1: nq x segments x k keys
    uint32_t* __restrict__ part_n;         // nq x segments counts
};

template <int kMetric>
__global__ void __launch_bounds__(kBfThreads) bf_scan_kernel(BfArgs a) {
    extern __shared__ __align__(16) unsigned char bf_smem[];
    uint64_t* lists = reinterpret_cast<uint64_t*>(bf_smem);                       // kBfQueries x list_cap
    float* qs = reinterpret_cast<float*>(lists + static_cast<size_t>(kBfQueries) * a.list_cap);  // kBfQueries x dim
    __shared__ uint32_t cnt[kBfQueries];
    __shared__ uint64_t thr[kBfQueries];
    __shared__ float qsq[kBfQueries];
    __shared__ int need;

    const uint32_t tid = threadIdx.x;
    const uint32_t q0 = blockIdx.x * kBfQueries;
    const uint32_t nqt = min(static_cast<uint32_t>(kBfQueries), a.nq - q0);
    const uint32_t dim = a.dim;
    for (uint32_t i = tid; i < kBfQueries * dim; i += kBfThreads) {
        const uint32_t qi = i / dim;
        qs[i] = qi < nqt ? a.queries[static_cast<size_t>(q0 + qi) * dim + (i - qi * dim)] : 0.0f;
    }
    if (tid < kBfQueries) {
        cnt[tid] = 0;
        thr[tid] = kMaxKey;
    }
    __syncthreads();
    if (kMetric == ARTEA_GPU_COSINE && tid < kBfQueries) {
        // The query's own lane chains (nsq1, simd_distance.hpp:251-268).
        float l[16];
        for (int j = 0; j < 16; ++j) l[j] = 0.0f;
        for (uint32_t c = 0; c < dim; c += 16)
            for (int j = 0; j < 16; ++j) l[j] = fmaf(qs[tid * dim + c + j], qs[tid * dim + c + j], l[j]);
        float t8[8], t4[4];
        for (int i = 0; i < 8; ++i) t8[i] = __fadd_rn(l[i], l[i + 8]);
        for (int i = 0; i < 4; ++i) t4[i] = __fadd_rn(t8[i], t8[i + 4]);
        qsq[tid] = __fadd_rn(__fadd_rn(t4[0], t4[2]), __fadd_rn(t4[1], t4[3]));
    }
    __syncthreads();

    const uint32_t r0 = blockIdx.y * a.seg_len;
    const uint32_t r1 = min(a.n_rows, r0 + a.seg_len);
    for (uint32_t base = r0; base < r1; base += kBfThreads) {
        const uint32_t r = base + tid;
        const bool valid = r < r1;
        const uint32_t vid = valid ? (a.subset ? a.subset[r] : r) : 0u;
        const float* row = a.vecs + static_cast<size_t>(vid) * dim;
        f32x2 A[kBfQueries][8];
        f32x2 B[8];
#pragma unroll
        for (int qi = 0; qi < kBfQueries; ++qi)
#pragma unroll
            for (int p = 0; p < 8; ++p) A[qi][p] = 0ull;
#pragma unroll
        for (int p = 0; p < 8; ++p) B[p] = 0ull;
        if (valid) {
            for (uint32_t c = 0; c < dim; c += 16) {
                f32x2 x[8];
                const ulonglong2* xr = reinterpret_cast<const ulonglong2*>(row + c);
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const ulonglong2 v = __ldg(xr + h);
                    x[2 * h] = v.x;
                    x[2 * h + 1] = v.y;
                }
                if (kMetric == ARTEA_GPU_COSINE) {
#pragma unroll
                    for (int p = 0; p < 8; ++p) B[p] = fma2(x[p], x[p], B[p]);
                }
#pragma unroll
                for (int qi = 0; qi < kBfQueries; ++qi) {
                    const ulonglong2* yr = reinterpret_cast<const ulonglong2*>(qs + qi * dim + c);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const ulonglong2 y = yr[h];
                        if (kMetric == ARTEA_GPU_EUCLIDEAN_SQR || kMetric == ARTEA_GPU_EUCLIDEAN) {
                            const f32x2 d0 = sub2(y.x, x[2 * h]), d1 = sub2(y.y, x[2 * h + 1]);
                            A[qi][2 * h] = fma2(d0, d0, A[qi][2 * h]);
                            A[qi][2 * h + 1] = fma2(d1, d1, A[qi][2 * h + 1]);
                        } else {
                            A[qi][2 * h] = fma2(y.x, x[2 * h], A[qi][2 * h]);
                            A[qi][2 * h + 1] = fma2(y.y, x[2 * h + 1], A[qi][2 * h + 1]);
                        }
                    }
                }
            }
        }
        float xsq = 0.0f;
        if (kMetric == ARTEA_GPU_COSINE) {
            float l[16];
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                l[2 * p] = lo32(B[p]);
                l[2 * p + 1] = hi32(B[p]);
            }
            float t8[8], t4[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) t8[i] = __fadd_rn(l[i], l[i + 8]);
#pragma unroll
            for (int i = 0; i < 4; ++i) t4[i] = __fadd_rn(t8[i], t8[i + 4]);
            xsq = __fadd_rn(__fadd_rn(t4[0], t4[2]), __fadd_rn(t4[1], t4[3]));
        }
#pragma unroll
        for (int qi = 0; qi < kBfQueries; ++qi) {
            float l[16];
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                l[2 * p] = lo32(A[qi][p]);
                l[2 * p + 1] = hi32(A[qi][p]);
            }
            float t8[8], t4[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) t8[i] = __fadd_rn(l[i], l[i + 8]);
#pragma unroll
            for (int i = 0; i < 4; ++i) t4[i] = __fadd_rn(t8[i], t8[i + 4]);
            float d = __fadd_rn(__fadd_rn(t4[0], t4[2]), __fadd_rn(t4[1], t4[3]));
            if (kMetric == ARTEA_GPU_EUCLIDEAN) {
                d = __fsqrt_rn(d);
            } else if (kMetric == ARTEA_GPU_DOT) {
                d = -d;
            } else if (kMetric == ARTEA_GPU_COSINE) {
                // utils/simd_distance.hpp:263-274
                const float denom = __fsqrt_rn(__fmul_rn(qsq[qi], xsq));
                d = denom > 0.0f ? __fsub_rn(1.0f, __fdiv_rn(d, denom)) : 1.0f;
            }
            if (valid && static_cast<uint32_t>(qi) < nqt) {
                const uint64_t key = order_key(d, vid);
                if (key < thr[qi]) {
                    const uint32_t pos = atomicAdd(&cnt[qi], 1u);
                    lists[static_cast<size_t>(qi) * a.list_cap + pos] = key;   // pos < list_cap: see below
                }
            }
        }
        __syncthreads();
        // A round appends at most kBfThreads keys per list; trim any list that
        // could overflow in the next round (list_cap >= k + 2 * kBfThreads).
        if (tid == 0) {
            int any = 0;
            for (int qi = 0; qi < kBfQueries; ++qi) any |= cnt[qi] > a.list_cap - kBfThreads;
            need = any;
        }
        __syncthreads();
        if (need) {
            const uint32_t warp = tid >> 5;
            for (uint32_t qi = warp; qi < static_cast<uint32_t>(kBfQueries); qi += kBfThreads / 32) {
                if (cnt[qi] > a.list_cap - kBfThreads)
                    trim_list(lists + static_cast<size_t>(qi) * a.list_cap, a.list_cap, &cnt[qi], &thr[qi], a.k);
            }
            __syncthreads();
        }
    }
    // Final trim of every list, then write words (one segment) or keys (several).
    const uint32_t warp = tid >> 5;
    for (uint32_t qi = warp; qi < nqt; qi += kBfThreads / 32)
        trim_list(lists + static_cast<size_t>(qi) * a.list_cap, a.list_cap, &cnt[qi], &thr[qi], a.k);
    __syncthreads();
    for (uint32_t qi = 0; qi < nqt; ++qi) {
        const uint64_t* l = lists + static_cast<size_t>(qi) * a.list_cap;
        const uint32_t n = cnt[qi];
        if (a.segments == 1) {
            uint64_t* o = a.out + static_cast<size_t>(q0 + qi) * a.k;
            for (uint32_t i = tid; i < a.k; i += kBfThreads) o[i] = i < n ? key_word(l[i]) : kDefaultEntryWord;
        } else {
            uint64_t* o = a.part + (static_cast<size_t>(q0 + qi) * a.segments + blockIdx.y) * a.k;
            for (uint32_t i = tid; i < n; i += kBfThreads) o[i] = l[i];
            if (tid == 0) a.part_n[static_cast<size_t>(q0 + qi) * a.segments + blockIdx.y] = n;
        }
    }
}

// One CTA per query: the best k of its segments' sorted key lists.
__global__ void __launch_bounds__(256) bf_merge_kernel(const uint64_t* __restrict__ part,
                                                       const uint32_t* __restrict__ part_n, uint32_t segments,
                                                       uint32_t k, uint32_t pow2, uint64_t* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char bf_smem[];
    uint64_t* keys = reinterpret_cast<uint64_t*>(bf_smem);   // pow2 >= segments * k
    const uint32_t q = blockIdx.x;
    for (uint32_t i = threadIdx.x; i < pow2; i += blockDim.x) keys[i] = kMaxKey;
    __syncthreads();
    for (uint32_t s = 0; s < segments; ++s) {
        const uint32_t n = part_n[static_cast<size_t>(q) * segments + s];
        const uint64_t* src = part + (static_cast<size_t>(q) * segments + s) * k;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) keys[s * k + i] = src[i];
    }
    __syncthreads();
    for (uint32_t k2 = 2; k2 <= pow2; k2 <<= 1) {
        for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < pow2; i += blockDim.x) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const uint64_t x = keys[i], y = keys[p];
                    if ((x > y) == ((i & k2) == 0)) {
                        keys[i] = y;
                        keys[p] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    uint64_t* o = out + static_cast<size_t>(q) * k;
    for (uint32_t i = threadIdx.x; i < k; i += blockDim.x)
        o[i] = keys[i] != kMaxKey ? key_word(keys[i]) : kDefaultEntryWord;
}

using ScanFn = void (*)(BfArgs);

ScanFn scan_kernel(int metric) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR: return bf_scan_kernel<ARTEA_GPU_EUCLIDEAN_SQR>;
        case ARTEA_GPU_EUCLIDEAN: return bf_scan_kernel<ARTEA_GPU_EUCLIDEAN>;
        case ARTEA_GPU_COSINE: return bf_scan_kernel<ARTEA_GPU_COSINE>;
        case ARTEA_GPU_DOT: return bf_scan_kernel<ARTEA_GPU_DOT>;
        default: return nullptr;
    }
}

// use_subset: rows are d_subset[0, n_subset) (possibly empty), else all vectors.
int bruteforce_impl(const artea_gpu_index* ix, int metric, const float* d_queries, uint32_t nq, uint32_t topk,
                    bool use_subset, const uint32_t* d_subset, uint32_t n_subset, uint64_t* d_out, cudaStream_t st) {
    if (!ix || (nq && (!d_queries || !d_out))) return fail(ARTEA_GPU_EINVAL, "null argument");
    if (topk == 0 || topk > kBfMaxTopk)
        return fail(ARTEA_GPU_EINVAL, "brute-force topk must be in [1, " + std::to_string(kBfMaxTopk) + "]");
    ScanFn fn = scan_kernel(metric);
    if (!fn) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    if (nq == 0) return ARTEA_GPU_OK;
    const uint32_t n_rows = use_subset ? n_subset : ix->nvecs;
    if (use_subset && n_subset && !d_subset) return fail(ARTEA_GPU_EINVAL, "null subset");
    DeviceGuard guard(ix->device);
    if (n_rows == 0) {
        // Every row is CandidateEntry() padding.
        std::vector<uint64_t> pad(static_cast<size_t>(nq) * topk, kDefaultEntryWord);
        CUDA_TRY(cudaMemcpyAsync(d_out, pad.data(), pad.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        return ARTEA_GPU_OK;
    }
    int dev_sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ix->device));
    const uint32_t list_cap = next_pow2(topk + 2 * kBfThreads);
    const size_t smem = static_cast<size_t>(kBfQueries) * list_cap * sizeof(uint64_t) +
                        static_cast<size_t>(kBfQueries) * ix->dim * sizeof(float);
    if (smem > 227u * 1024u) return fail(ARTEA_GPU_EINVAL, "brute-force tile exceeds shared memory (topk or dim too large)");
    CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(fn), kBfThreads,
                                                           smem));
    const uint32_t tiles = (nq + kBfQueries - 1) / kBfQueries;
    // Split the rows into segments until the grid covers the GPU twice over,
    // keeping each segment >= 4096 rows and the merge within shared memory.
    const uint32_t want = 2u * static_cast<uint32_t>(std::max(per_sm, 1) * dev_sms);
    uint32_t segments = std::max(1u, (want + tiles - 1) / tiles);
    segments = std::min(segments, std::max(1u, n_rows / 4096u));
    segments = std::min(segments, std::max(1u, 16384u / topk));
    const uint32_t seg_len = (n_rows + segments - 1) / segments;
    segments = (n_rows + seg_len - 1) / seg_len;

    BfArgs a;
    std::memset(&a, 0, sizeof(a));
    a.vecs = ix->d_vecs;
    a.dim = ix->dim;
    a.subset = use_subset ? d_subset : nullptr;
    a.n_rows = n_rows;
    a.queries = d_queries;
    a.nq = nq;
    a.k = topk;
    a.seg_len = seg_len;
    a.segments = segments;
    a.list_cap = list_cap;
    a.out = d_out;
    uint64_t* part = nullptr;
    uint32_t* part_n = nullptr;
    if (segments > 1) {
        if (int rc = dev_alloc(&part, static_cast<size_t>(nq) * segments * topk)) return rc;
        if (int rc = dev_alloc(&part_n, static_cast<size_t>(nq) * segments)) {
            dev_free(part);
            return rc;
        }
        a.part = part;
        a.part_n = part_n;
    }
    fn<<<dim3(tiles, segments), kBfThreads, smem, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && segments > 1) {
        const uint32_t pow2 = next_pow2(segments * topk);
        const size_t msmem = static_cast<size_t>(pow2) * sizeof(uint64_t);
        e = cudaFuncSetAttribute(reinterpret_cast<const void*>(bf_merge_kernel),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(msmem));
        if (e == cudaSuccess) {
            bf_merge_kernel<<<nq, 256, msmem, st>>>(part, part_n, segments, topk, pow2, d_out);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dev_free(part);
    dev_free(part_n);
    if (e != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string("brute force: ") + cudaGetErrorString(e));
    return ARTEA_GPU_OK;
}

// Centroid of the bucket's rows (hierarchical_graph_compactor.hpp:261-300):
// block b sums rows [b * rows_per_block, ...) of every dimension in double,
// in row order; the final pass adds the blocks' sums in block order.
__global__ void centroid_partial_kernel(const float* __restrict__ vecs, uint32_t dim,
                                        const uint32_t* __restrict__ bucket, uint32_t n, uint32_t rows_per_block,
                                        double* __restrict__ partial) {
    const uint32_t r0 = blockIdx.x * rows_per_block;
    const uint32_t r1 = min(n, r0 + rows_per_block);
    for (uint32_t d = threadIdx.x; d < dim; d += blockDim.x) {
        double s = 0.0;
        for (uint32_t r = r0; r < r1; ++r) {
            const uint32_t vid = bucket ? bucket[r] : r;
            s += static_cast<double>(vecs[static_cast<size_t>(vid) * dim + d]);
        }
        partial[static_cast<size_t>(blockIdx.x) * dim + d] = s;
    }
}

__global__ void centroid_final_kernel(const double* __restrict__ partial, uint32_t blocks, uint32_t dim, uint32_t n,
                                      float* __restrict__ centroid) {
    const double inv_n = 1.0 / static_cast<double>(n);
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < dim; d += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < blocks; ++b) s += partial[static_cast<size_t>(b) * dim + d];
        centroid[d] = static_cast<float>(s * inv_n);
    }
}

}  // namespace
}  // namespace artea_gpu

using namespace artea_gpu;

extern "C" {

int artea_gpu_bruteforce_device(const artea_gpu_index* index, int metric, const float* d_queries, uint32_t nq,
                                uint32_t topk, const uint32_t* d_subset, uint32_t n_subset, uint64_t* d_out,
                                void* stream) {
    return bruteforce_impl(index, metric, d_queries, nq, topk, d_subset != nullptr, d_subset, n_subset, d_out,
                           static_cast<cudaStream_t>(stream));
}

int artea_gpu_bruteforce(const artea_gpu_index* index, int metric, const float* queries, uint32_t nq, uint32_t topk,
                         const uint32_t* subset, uint32_t n_subset, uint64_t* out) {
    if (!index || (nq && (!queries || !out))) return fail(ARTEA_GPU_EINVAL, "null argument");
    if (subset) {
        for (uint32_t i = 0; i < n_subset; ++i)
            if (subset[i] >= index->nvecs)
                return fail(ARTEA_GPU_EINVAL, "subset id " + std::to_string(subset[i]) + " out of range");
    }
    if (nq == 0) return ARTEA_GPU_OK;
    DeviceGuard guard(index->device);
    float* d_q = nullptr;
    uint64_t* d_o = nullptr;
    uint32_t* d_s = nullptr;
    int rc = dev_alloc(&d_q, static_cast<size_t>(nq) * index->dim);
    if (!rc) rc = dev_alloc(&d_o, static_cast<size_t>(nq) * topk);
    if (!rc && subset && n_subset) rc = dev_alloc(&d_s, n_subset);
    if (!rc && cudaMemcpy(d_q, queries, sizeof(float) * nq * index->dim, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(ARTEA_GPU_ECUDA, "query upload failed");
    if (!rc && d_s && cudaMemcpy(d_s, subset, sizeof(uint32_t) * n_subset, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(ARTEA_GPU_ECUDA, "subset upload failed");
    if (!rc) rc = bruteforce_impl(index, metric, d_q, nq, topk, subset != nullptr, d_s, subset ? n_subset : 0u, d_o,
                                  nullptr);
    if (!rc && cudaMemcpy(out, d_o, sizeof(uint64_t) * nq * topk, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail(ARTEA_GPU_ECUDA, "result download failed");
    dev_free(d_q);
    dev_free(d_o);
    dev_free(d_s);
    return rc;
}

// _compute_entry_point_vid (hierarchical_graph_compactor.hpp:261-327): the
// bucket's centroid (double sums, rounded to float), then the bucket vid
// nearest to it under metric -- the brute force above with k = 1 over the
// bucket, the centroid as the query operand.
int artea_gpu_centroid_entry(const artea_gpu_index* index, int metric, const uint32_t* bucket, uint32_t n,
                             uint32_t* out_vid) {
    if (!index || !out_vid) return fail(ARTEA_GPU_EINVAL, "null argument");
    const uint32_t rows = bucket ? n : index->nvecs;
    *out_vid = 0xFFFFFFFFu;   // invalid_vertex_id: empty bucket
    if (rows == 0) return ARTEA_GPU_OK;
    if (bucket) {
        for (uint32_t i = 0; i < n; ++i)
            if (bucket[i] >= index->nvecs)
                return fail(ARTEA_GPU_EINVAL, "bucket id " + std::to_string(bucket[i]) + " out of range");
    }
    DeviceGuard guard(index->device);
    const uint32_t per_block = 4096;
    const uint32_t blocks = (rows + per_block - 1) / per_block;
    uint32_t* d_bucket = nullptr;
    double* d_partial = nullptr;
    float* d_centroid = nullptr;
    uint64_t* d_word = nullptr;
    int rc = dev_alloc(&d_partial, static_cast<size_t>(blocks) * index->dim);
    if (!rc) rc = dev_alloc(&d_centroid, index->dim);
    if (!rc) rc = dev_alloc(&d_word, 1);
    if (!rc && bucket) {
        rc = dev_alloc(&d_bucket, n);
        if (!rc && cudaMemcpy(d_bucket, bucket, sizeof(uint32_t) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(ARTEA_GPU_ECUDA, "bucket upload failed");
    }
    if (!rc) {
        centroid_partial_kernel<<<blocks, 256>>>(index->d_vecs, index->dim, d_bucket, rows, per_block, d_partial);
        centroid_final_kernel<<<(index->dim + 255) / 256, 256>>>(d_partial, blocks, index->dim, rows, d_centroid);
        if (cudaGetLastError() != cudaSuccess) rc = fail(ARTEA_GPU_ECUDA, "centroid kernels failed to launch");
    }
    if (!rc) rc = bruteforce_impl(index, metric, d_centroid, 1, 1, bucket != nullptr, d_bucket, rows, d_word, nullptr);
    uint64_t word = 0;
    if (!rc && cudaMemcpy(&word, d_word, sizeof(word), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail(ARTEA_GPU_ECUDA, "result download failed");
    if (!rc) *out_vid = static_cast<uint32_t>(word);
    dev_free(d_bucket);
    dev_free(d_partial);
    dev_free(d_centroid);
    dev_free(d_word);
    return rc;
}

}  // extern "C"
