// Device side of the B200 query path: one warp searches one query.
//
// Restates, on the GPU, hierarchical_graph_router.hpp:195-248 (_query with
// RandomSeeding=false; enable_early_stop either way): entry point, greedy descent
// on levels top..1 (detail/beam_loop.hpp:129-166), beam search on level 0
// (detail/beam_loop.hpp:90-119) with StdCandidateQueue's rules
// (router/data_structures/std_candidate_queue.hpp:358-513), top-k extraction
// (std_candidate_queue.hpp:542-561).
//
// Data layout in HBM (uploaded once):
//   vecs      N x D float32, D a multiple of 16, rows 64-byte aligned
//   vinfo     N x {highest_level, local_vid} (uint2)
//   offsets   per highest-level group h: N_h*(h+1)+1 uint64 CSR offsets
//   nbrs      uint32 neighbour ids in CSR row order
//   l0row     N x uint64 level-0 row descriptor: start | length << 40
// Per search slot (one per resident warp): a spill bitset (N bits) and the
// list of ids set in it since the last clear.
//
// Shared memory per warp: the query row, the candidate queue (sorted array of
// (dist, vid|explored), 2L slots), a candidate batch and the visited hash.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

#include "../../include/artea_gpu.h"

namespace artea_gpu {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kExplored = 0x80000000u;
constexpr uint32_t kVidMask = 0x7fffffffu;
constexpr uint32_t kInvalidLevel = 0xffffffffu;
constexpr uint32_t kEmptySlot = 0xffffffffu;
constexpr uint32_t kCandBatch = 64;     // candidates evaluated per distance batch
constexpr int kMaxGroups = 64;
constexpr int kRowLenShift = 40;        // l0row: start in bits 0..39, length in 40..63
constexpr unsigned long long kRowStartMask = (1ull << kRowLenShift) - 1ull;

enum : int {
    kErrNone = 0,
    kErrBadVid = 1,        // an id >= N reached the kernel
    kErrBound = 2,         // an iteration bound was exceeded
    kErrQueue = 3,         // queue capacity exceeded (cannot happen for cap >= 2L)
    kErrArgs = 4,          // per-query topk/queue outside the launch's limits
    kErrTimeout = 5,       // a bulk copy did not complete within the wait bound
};

constexpr uint32_t kStageRows = 8;          // rows per staged pass (one per row group)
constexpr uint32_t kStagePad = 4;           // words of padding per staged row (bank spread)
constexpr uint32_t kWaitBound = 1u << 22;   // mbarrier polls before a copy counts as lost

struct DeviceGraph {
    const float* __restrict__ vecs;
    const float* __restrict__ xsq;   // per-row x.x (row_sqnorm_kernel)
    const uint2* __restrict__ vinfo;
    const uint32_t* __restrict__ nbrs;
    const unsigned long long* __restrict__ l0row;
    uint32_t n;
    uint32_t dim;
    uint32_t top;      // kInvalidLevel when empty
    uint32_t entry;
    uint32_t l0_unique;   // every level-0 row of <= 64 ids holds distinct ids
    const uint64_t* offsets[kMaxGroups];
};

// Trace of a search for the subsystem probes (kernels compiled with kTrace):
// per query, the level-0 expansions (vid, new candidates), the candidates'
// ids and distances in evaluation order, the cursor that seeds level 0, and
// the lengths recorded (capped at cap / rows_cap).
struct TraceArgs {
    uint32_t* ids;       // nq x cap
    float* dists;        // nq x cap
    uint2* rows;         // nq x rows_cap: (expanded vid, new candidates)
    uint2* cur;          // nq: (cursor vid, its distance bits)
    uint2* len;          // nq: (candidates, rows) recorded
    uint32_t cap;
    uint32_t rows_cap;
    uint32_t upper_only; // stop after the upper levels (the greedy descent alone)
};

struct SearchArgs {
    DeviceGraph g;
    const float* __restrict__ queries;
    uint32_t nq;
    const uint32_t* __restrict__ topk;    // may be null
    const uint32_t* __restrict__ queue;   // may be null
    uint32_t topk_default;
    uint32_t queue_default;
    uint32_t k_stride;
    uint32_t cap;                         // queue entries per warp (>= 2 * max queue)
    uint32_t vh_bits;                     // log2 of the shared-memory visited table in 16-byte units (0: none)
    uint32_t vk_bits;                     // log2 of the vid permutation space (visited_kbits)
    uint64_t* __restrict__ out;
    artea_gpu_query_stats* __restrict__ stats;   // may be null
    uint32_t* __restrict__ vis_bits;      // slots x words_per_slot
    uint32_t* __restrict__ vis_list;      // slots x list_cap
    uint64_t words_per_slot;
    uint32_t list_cap;
    uint32_t* __restrict__ next_query;    // persistent schedule work counter
    int* __restrict__ error;
    uint32_t l0_only;
    unsigned long long* __restrict__ phase_cycles;   // nq x kPhases, optional
    uint32_t coherent;        // queries/topk/queue may change while the kernel runs (serving ring)
    uint32_t early_stop;      // stop level-h greedy walks at distance <= es_thr[h]
    float es_thr[kMaxGroups]; // per-level thresholds in query distance units
    uint32_t compact;         // queue capacity may be below 2L: a query that could lose a live
                              // entry is abandoned and listed in overflow for the full-capacity rerun
    uint32_t* __restrict__ overflow;   // [count, rerun counter, query indices...] (compact only)
    uint32_t l0_pipe;         // level-0 rows hold <= 64 distinct ids: pipelined level-0 loop
    uint32_t pf_l2;           // pipelined loop: also prefetch the second pass's rows into L2
    const uint32_t* __restrict__ order;   // persistent schedule: query order (null: 0..nq-1)
    TraceArgs tr;             // kernels compiled with kTrace only
};

// Phase-cycle breakdown written per query when phase_cycles is set.
enum : int {
    kPhUpper = 0,     // greedy descent on levels >= 1
    kPhPop = 1,       // pop, row descriptor, first ids, next-entry prefetch
    kPhCollect = 2,   // row ids + visited test_and_set
    kPhDist = 3,      // distance batches
    kPhMerge = 4,     // queue merge
    kPhTail = 5,      // result write-out and visited clear
    kPhTotal = 6,     // whole query
    kPhPrefetchHits = 7,  // expansions whose row descriptor was prefetched
    kPhases = 8
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ bool entry_less(float da, uint32_t va, float db, uint32_t vb) {
    return da < db || (da == db && (va & kVidMask) < (vb & kVidMask));
}

__device__ __forceinline__ void set_error(int* error, int code) {
    atomicCAS(error, 0, code);
}

// ---------------------------------------------------------------------------
// Distances (subsystem d). 4 lanes per row, 8 rows per warp pass. Lane group
// slot g in [0,4) owns AVX-512 lanes 4g..4g+3 of the reference's 16-lane
// accumulation (utils/simd_distance.hpp:100-115): for chunk c it loads the
// float4 at element 16c+4g and FMAs into four accumulators, so each
// accumulator is exactly one reference lane's chain. The fold then follows
// GCC's _mm512_reduce_add_ps tree: lanes (i, i+8) are warp lanes g and g^2,
// lanes (i, i+4) are g and g^1, then (i, i^2) and lane0+lane1 inside a lane.
// FAST mode folds each lane's four components first (warp order).
// ---------------------------------------------------------------------------
template <bool kExact>
__device__ __forceinline__ float fold16(float a0, float a1, float a2, float a3) {
    if (kExact) {
        a0 = __fadd_rn(a0, __shfl_xor_sync(kFull, a0, 2));
        a1 = __fadd_rn(a1, __shfl_xor_sync(kFull, a1, 2));
        a2 = __fadd_rn(a2, __shfl_xor_sync(kFull, a2, 2));
        a3 = __fadd_rn(a3, __shfl_xor_sync(kFull, a3, 2));
        a0 = __fadd_rn(a0, __shfl_xor_sync(kFull, a0, 1));
        a1 = __fadd_rn(a1, __shfl_xor_sync(kFull, a1, 1));
        a2 = __fadd_rn(a2, __shfl_xor_sync(kFull, a2, 1));
        a3 = __fadd_rn(a3, __shfl_xor_sync(kFull, a3, 1));
        const float u0 = __fadd_rn(a0, a2);
        const float u1 = __fadd_rn(a1, a3);
        return __fadd_rn(u0, u1);
    } else {
        float s = (a0 + a1) + (a2 + a3);
        s += __shfl_xor_sync(kFull, s, 1);
        s += __shfl_xor_sync(kFull, s, 2);
        return s;
    }
}

__device__ __forceinline__ float4 ldg4(const float* p) {
    return __ldg(reinterpret_cast<const float4*>(p));
}

// Squared norm of the query with the reference's lane structure (the nsq1
// accumulator of utils/simd_distance.hpp:251-268), needed by cosine.
template <bool kExact>
__device__ float query_sqnorm(const float* __restrict__ q, uint32_t dim) {
    const int g = lane_id() & 3;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    for (uint32_t c = 0; c < dim; c += 16) {
        const float4 v = *reinterpret_cast<const float4*>(q + c + 4 * g);
        a0 = fmaf(v.x, v.x, a0); a1 = fmaf(v.y, v.y, a1);
        a2 = fmaf(v.z, v.z, a2); a3 = fmaf(v.w, v.w, a3);
    }
    return fold16<kExact>(a0, a1, a2, a3);
}

// Per pass each lane issues up to kBlock float4 loads of its row segment
// before any arithmetic, so a D=128 row costs one memory round trip.
constexpr int kBlock = 8;

// Packed FP32x2 arithmetic (sm_100): each element is rounded on its own, as
// two scalar instructions would round it, so the exact mode is unaffected;
// the pair halves the instruction count of the accumulation.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ float lo32(f32x2 v) { return __uint_as_float(static_cast<uint32_t>(v)); }
__device__ __forceinline__ float hi32(f32x2 v) { return __uint_as_float(static_cast<uint32_t>(v >> 32)); }

// One chunk of 4 elements (x from the row, y from the query) into the pair
// accumulators A01/A23.
template <int kMetric>
__device__ __forceinline__ void accumulate(const ulonglong2 x, const ulonglong2 y, f32x2& A01, f32x2& A23) {
    if (kMetric == ARTEA_GPU_EUCLIDEAN_SQR || kMetric == ARTEA_GPU_EUCLIDEAN) {
        const f32x2 d01 = sub2(y.x, x.x), d23 = sub2(y.y, x.y);
        A01 = fma2(d01, d01, A01);
        A23 = fma2(d23, d23, A23);
    } else {
        // dot and cosine: q.x (cosine's x.x comes from the index's row norms)
        A01 = fma2(y.x, x.x, A01);
        A23 = fma2(y.y, x.y, A23);
    }
}

// ---------------------------------------------------------------------------
// TMA row staging: one cp.async.bulk per candidate row into the warp's
// shared-memory stage, completion counted on the warp's mbarrier, so a pass
// costs one memory round trip whatever the row length.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_row_copy(uint32_t dst, const float* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

// Bounded wait for the phase with the given parity; false if it never came.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitBound; ++i) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

struct Stage {
    float* buf;          // kStageRows rows of dim + kStagePad words (null: no staging)
    uint32_t mbar;       // shared address of the warp's mbarrier
    uint32_t phase;      // parity of the next phase to wait for
};

// Loads of the next expansion's rows, issued ahead of its distance phase so
// they are in flight while the warp merges the current batch. With kRegs, the
// first pass's first block of chunks (rows cvid[0, 8), one float4 per chunk
// and lane) is loaded into x, which batch_distances then consumes (kPre);
// without, those rows' first 512 bytes are prefetched into L2 (one 128-byte
// line per lane). With l2_next, the second pass's rows (cvid[8, 16)) are
// prefetched into L2 as well.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <bool kRegs>
__device__ __forceinline__ void dist_preload(const DeviceGraph& g, const uint32_t* cvid, uint32_t cnt,
                                             ulonglong2 (&x)[kBlock], bool l2_next) {
    const int lane = lane_id();
    const uint32_t r = static_cast<uint32_t>(lane) >> 2;
    const uint32_t gi = lane & 3;
    const uint32_t dim = g.dim;
    const uint32_t off = 128u * gi;   // byte offset of this lane's line in a row
    if (kRegs) {
        const uint32_t nchunks = dim >> 4;
        const bool valid = r < cnt;
        const uint32_t vid = valid ? cvid[r] : 0u;
        const float* row = g.vecs + static_cast<size_t>(vid) * dim + 4 * gi;
#pragma unroll
        for (int k = 0; k < kBlock; ++k) {
            const ulonglong2* src = reinterpret_cast<const ulonglong2*>(row + 16 * k);
            x[k] = (valid && static_cast<uint32_t>(k) < nchunks) ? __ldg(src) : make_ulonglong2(0ull, 0ull);
        }
    } else if (r < cnt && off < dim * 4u) {
        prefetch_l2(reinterpret_cast<const char*>(g.vecs + static_cast<size_t>(cvid[r]) * dim) + off);
    }
    if (l2_next && cnt > 8u) {
        const uint32_t r2 = 8u + r;
        if (r2 < cnt && off < dim * 4u)
            prefetch_l2(reinterpret_cast<const char*>(g.vecs + static_cast<size_t>(cvid[r2]) * dim) + off);
    }
}

// Distances for cnt candidates (ids in cvid, shared memory) into cdist, one
// pass of 8 rows at a time: passes pass0, pass0 + stride, ... (the warps of a
// cooperative search split the passes; one warp alone takes them all). With
// kPre, the first pass's first block of chunks is taken from pre (loaded by
// dist_preload<true> on the same cvid) instead of being loaded here.
template <int kMetric, bool kExact, bool kStage, bool kPre = false, bool kSplit = false>
__device__ void batch_distances(const DeviceGraph& g, const float* __restrict__ q, float qsq,
                                const uint32_t* cvid, float* cdist, uint32_t cnt, Stage& st, int* error,
                                const ulonglong2 (*pre)[kBlock] = nullptr, uint32_t pass0 = 0,
                                uint32_t stride = 1) {
    if (!kSplit) {
        pass0 = 0;
        stride = 1;
    }
    const int lane = lane_id();
    const int r = lane >> 2;
    const int gi = lane & 3;
    const uint32_t dim = g.dim;
    const uint32_t nchunks = dim >> 4;
    const uint32_t sstride = dim + kStagePad;
    for (uint32_t p = 8u * pass0; p < cnt; p += 8u * stride) {
        const uint32_t idx = p + r;
        const bool valid = idx < cnt;
        const uint32_t vid = valid ? cvid[idx] : 0u;
        // x.x of the row, stored at index creation in this kernel's exact
        // summation order (row_sqnorm_kernel); loaded ahead of the row.
        const float xsq = (kMetric == ARTEA_GPU_COSINE && valid) ? __ldg(g.xsq + vid) : 1.0f;
        const float* row;
        if (kStage) {
            // The stage's previous contents have been read by every lane
            // (generic proxy) before the async proxy overwrites them.
            const uint32_t nrows = min(kStageRows, cnt - p);
            __syncwarp();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (lane == 0) mbar_expect(st.mbar, nrows * dim * 4u);
            __syncwarp();
            if (static_cast<uint32_t>(lane) < nrows)
                bulk_row_copy(smem_addr(st.buf + lane * sstride), g.vecs + static_cast<size_t>(cvid[p + lane]) * dim,
                              dim * 4u, st.mbar);
            if (!mbar_wait(st.mbar, st.phase)) {
                set_error(error, kErrTimeout);
                mbar_wait(st.mbar, st.phase);   // a second bounded wait for the copies in flight
            }
            st.phase ^= 1u;
            row = st.buf + r * sstride + 4 * gi;
        } else {
            row = g.vecs + static_cast<size_t>(vid) * dim + 4 * gi;
        }
        const float* qq = q + 4 * gi;
        f32x2 A01 = 0ull, A23 = 0ull;   // L2: diff^2; dot/cos: q*x   (+0.0f pairs)
        for (uint32_t cb = 0; cb < nchunks; cb += kBlock) {
            ulonglong2 x[kBlock];
            if (kPre && p == 0 && cb == 0) {
#pragma unroll
                for (int k = 0; k < kBlock; ++k) x[k] = (*pre)[k];
            } else {
#pragma unroll
                for (int k = 0; k < kBlock; ++k) {
                    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(row + 16 * (cb + k));
                    x[k] = (valid && cb + k < nchunks) ? (kStage ? *src : __ldg(src)) : make_ulonglong2(0ull, 0ull);
                }
            }
#pragma unroll
            for (int k = 0; k < kBlock; ++k) {
                if (cb + k < nchunks) {
                    const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(qq + 16 * (cb + k));
                    accumulate<kMetric>(x[k], y, A01, A23);
                }
            }
        }
        const float a0 = lo32(A01), a1 = hi32(A01), a2 = lo32(A23), a3 = hi32(A23);
        float res = fold16<kExact>(a0, a1, a2, a3);
        if (kMetric == ARTEA_GPU_EUCLIDEAN) {
            res = __fsqrt_rn(res);
        } else if (kMetric == ARTEA_GPU_DOT) {
            res = -res;
        } else if (kMetric == ARTEA_GPU_COSINE) {
            // utils/simd_distance.hpp:263-274
            const float denom = __fsqrt_rn(__fmul_rn(qsq, xsq));
            res = denom > 0.0f ? __fsub_rn(1.0f, __fdiv_rn(res, denom)) : 1.0f;
        }
        if (valid && gi == 0) cdist[idx] = res;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Cooperative distances (warps per query > 1). A CTA of kW warps searches one
// query: warp 0 runs the search; at every distance batch it publishes the
// candidates here and all kW warps take the 8-row passes in turn (warp w:
// passes w, w + kW, ...), each row by one warp with the same code, so the
// distances are bit-identical to one warp's. Two named-barrier phases per
// batch: start (the batch is published) and done (every distance is
// written). After its last query warp 0 publishes quit at a start barrier.
// ---------------------------------------------------------------------------
struct CoopCtl {
    const uint32_t* cvid;
    float* cdist;
    uint32_t cnt;
    float qsq;
    uint32_t quit;
    uint32_t pad[3];
};
constexpr uint32_t kCoopWords = sizeof(CoopCtl) / 4;
constexpr int kCoopBarrier = 1;

__device__ __forceinline__ void coop_barrier(int warps) {
    asm volatile("barrier.sync %0, %1;" ::"r"(kCoopBarrier), "r"(warps * 32) : "memory");
}

template <int kMetric, bool kExact, bool kStage, int kW>
__device__ __forceinline__ void dist_call(const DeviceGraph& g, const float* __restrict__ q, float qsq,
                                          const uint32_t* cvid, float* cdist, uint32_t cnt, Stage& st, int* error,
                                          CoopCtl* coop) {
    if (kW == 1) {
        batch_distances<kMetric, kExact, kStage>(g, q, qsq, cvid, cdist, cnt, st, error);
        return;
    }
    if (lane_id() == 0) {
        coop->cvid = cvid;
        coop->cdist = cdist;
        coop->cnt = cnt;
        coop->qsq = qsq;
        coop->quit = 0u;
    }
    coop_barrier(kW);   // start
    batch_distances<kMetric, kExact, false, false, true>(g, q, qsq, cvid, cdist, cnt, st, error, nullptr, 0u, kW);
    coop_barrier(kW);   // done
}

// The other warps of a cooperative CTA: take passes of each published batch
// until warp 0 publishes quit.
template <int kMetric, bool kExact, int kW>
__device__ void coop_helper(const DeviceGraph& g, const float* __restrict__ q, CoopCtl* coop, int warp, int* error) {
    Stage st;
    st.buf = nullptr;
    st.mbar = 0u;
    st.phase = 0u;
    for (;;) {
        coop_barrier(kW);   // start
        const uint32_t quit = coop->quit;
        const uint32_t cnt = coop->cnt;
        const uint32_t* cvid = coop->cvid;
        float* cdist = coop->cdist;
        const float qsq = coop->qsq;
        if (quit) break;
        batch_distances<kMetric, kExact, false, false, true>(g, q, qsq, cvid, cdist, cnt, st, error, nullptr,
                                                            static_cast<uint32_t>(warp), kW);
        coop_barrier(kW);   // done
    }
}

// ---------------------------------------------------------------------------
// Visited set (subsystem c): exact, in two tiers.
//   1. A bucketed table in shared memory. vid -> p = (vid * odd) mod 2^kbits is
//      a bijection, so (bucket A = high tbits bits of p, quotient Q = the other
//      kbits - tbits bits) identifies vid exactly; a bucket is 4 uint16 slots
//      (8 bytes, one load), 0xFFFF marks an empty slot. When the quotient has
//      at most 14 bits, an id whose bucket A is full goes to a second bucket
//      B = A ^ alt(Q), stored as Q | 0x8000: the flag keeps it apart from
//      B's own ids (whose slots hold flag-free quotients), and B with Q gives
//      back A and so the id. Buckets only fill up, never drain, until clear():
//      an id absent from A while A has a free slot was never visited (it would
//      only have gone to B with A full), likewise for B.
//   2. The slot's bitset in HBM (atomicOr = test_and_set,
//      containers/version_tag_table.hpp:128-132), used for ids whose buckets
//      are full.
// Ids set in the bitset are listed so clear() (a version bump in the
// reference, version_tag_table.hpp:142-148) zeroes only the words it touched,
// or the whole bitset if the list overflowed. With no table (tbits == 0)
// every id goes to the bitset.
// ---------------------------------------------------------------------------
constexpr uint32_t kVisitedMul = 0x9E3779B1u;   // odd: multiplication mod 2^k is a bijection
constexpr uint32_t kAltFlag = 0x8000u;          // slot holds an id whose first bucket was full

// Permutation space of the table for a graph of n vertices and a table of
// 16 << table_log bytes (2^(table_log + 1) buckets of 8 bytes): returns kbits
// (>= log2 n and > the bucket bits), or 0 when a quotient would not fit in
// 15 bits (table too small for n).
__host__ __device__ inline uint32_t visited_kbits(uint32_t n, uint32_t table_log) {
    uint32_t kb = 1;
    while (kb < 32 && (1ull << kb) < n) ++kb;
    if (table_log == 0) return kb;
    const uint32_t tbits = table_log + 1;
    if (kb < tbits + 1) kb = tbits + 1;
    return kb - tbits > 15 ? 0u : kb;
}

struct Visited {
    uint2* tab;         // shared-memory buckets (4 uint16 slots each)
    uint32_t tbits;     // log2 of the bucket count (0: no table)
    uint32_t kbits;     // log2 of the permutation space
    uint32_t kmask;     // 2^kbits - 1
    uint32_t* bits;
    uint32_t* list;
    uint32_t list_n;
    uint32_t list_cap;
    uint64_t words;
    bool global_used;
    bool list_overflow;
    uint32_t spills;
};

// One id's place in the table: its first bucket, its second (~0u when the
// quotient leaves no second choice) and its quotient.
struct TableWalk {
    uint32_t a;
    uint32_t b;
    uint32_t q;
};

__device__ __forceinline__ TableWalk table_walk(const Visited& vs, uint32_t vid) {
    const uint32_t p = (vid * kVisitedMul) & vs.kmask;
    const uint32_t qbits = vs.kbits - vs.tbits;
    TableWalk w;
    w.a = p >> qbits;
    w.q = p & ((1u << qbits) - 1u);
    // alt(Q): the second bucket's offset from the quotient's bits (0 would
    // give B == A: no second choice for that quotient).
    const uint32_t h = (w.q * 0x2545F491u) >> (32u - vs.tbits);
    w.b = (qbits <= 14 && h != 0) ? (w.a ^ h) : 0xffffffffu;
    return w;
}

// Both buckets read at once (at most one CAS): 1 if the id is present (Q in
// A, or Q | flag in B), 0 if it was inserted now (into A while A has a free
// slot, else into B), 2 if both are full (the bitset decides), -1 if another
// lane filled the chosen slot meanwhile (read again). A match in B is the id
// itself whatever A holds: (B, Q) gives back A.
__device__ __forceinline__ int table_try(const Visited& vs, const TableWalk& w) {
    const bool has_b = w.b != 0xffffffffu;
    const uint2 ba = vs.tab[w.a];
    const uint2 bb = has_b ? vs.tab[w.b] : make_uint2(0u, 0u);   // no empty slot, no flagged value
    const uint32_t fq = w.q | kAltFlag;
    const uint32_t pa = w.q | (w.q << 16), pb = fq | (fq << 16);
    if (__vcmpeq2(ba.x, pa) | __vcmpeq2(ba.y, pa) | __vcmpeq2(bb.x, pb) | __vcmpeq2(bb.y, pb)) return 1;
    uint32_t e0 = __vcmpeq2(ba.x, 0xFFFFFFFFu), e1 = __vcmpeq2(ba.y, 0xFFFFFFFFu);
    uint32_t bucket = w.a, val = w.q;
    uint2 bk = ba;
    if (!(e0 | e1)) {
        // A is full (for good): B decides.
        e0 = __vcmpeq2(bb.x, 0xFFFFFFFFu);
        e1 = __vcmpeq2(bb.y, 0xFFFFFFFFu);
        if (!(e0 | e1)) return 2;
        bucket = w.b;
        val = fq;
        bk = bb;
    }
    const int wi = e0 ? 0 : 1;
    const uint32_t old = e0 ? bk.x : bk.y;
    const uint32_t e = e0 ? e0 : e1;
    const uint32_t desired = (e & 0xFFFFu) ? ((old & 0xFFFF0000u) | val) : ((old & 0x0000FFFFu) | (val << 16));
    uint32_t* word = reinterpret_cast<uint32_t*>(vs.tab + bucket) + wi;
    return atomicCAS(word, old, desired) == old ? 0 : -1;
}

// Returns 1 if vid is in the table, 0 if it was inserted now, 2 if its
// buckets are full (the bitset decides). Every retry follows a slot filled
// by another lane, so the loop ends within the 8 slots of the two buckets.
__device__ __forceinline__ int table_test_insert(const Visited& vs, uint32_t vid) {
    const TableWalk w = table_walk(vs, vid);
    for (int step = 0; step < 24; ++step) {
        const int r = table_try(vs, w);
        if (r >= 0) return r;
    }
    return 2;
}

// test_and_set for one id per lane (act lanes hold distinct vids); all lanes
// call. Returns true in the lanes whose id was not yet visited.
__device__ __forceinline__ bool visited_test_and_set(Visited& vs, uint32_t vid, bool act) {
    const int lane = lane_id();
    bool is_new = false;
    bool in_bits = false;
    if (act) {
        const int t = vs.tbits ? table_test_insert(vs, vid) : 2;
        if (t == 0) {
            is_new = true;
        } else if (t == 2) {
            const uint32_t mask = 1u << (vid & 31);
            const uint32_t old = atomicOr(vs.bits + (vid >> 5), mask);
            is_new = !(old & mask);
            in_bits = is_new;
        }
    }
    const uint32_t b = __ballot_sync(kFull, in_bits);
    if (b) {
        const uint32_t pos = vs.list_n + __popc(b & ((1u << lane) - 1u));
        if (in_bits && pos < vs.list_cap) vs.list[pos] = vid;
        const uint32_t total = vs.list_n + __popc(b);
        if (total > vs.list_cap) vs.list_overflow = true;
        vs.list_n = min(total, vs.list_cap);
        vs.global_used = true;
    }
    __syncwarp();
    return is_new;
}

// set(): mark one id (all lanes call with the same vid).
__device__ __forceinline__ void visited_set(Visited& vs, uint32_t vid) {
    visited_test_and_set(vs, vid, lane_id() == 0);
}

// table_test_insert for two distinct ids per lane, the two walks
// interleaved. r0/r1 as table_test_insert's return values (-1: inactive).
__device__ __forceinline__ void table_test_insert2(const Visited& vs, uint32_t v0, bool a0, uint32_t v1, bool a1,
                                                   int* r0, int* r1) {
    const TableWalk w0 = table_walk(vs, a0 ? v0 : 0u), w1 = table_walk(vs, a1 ? v1 : 0u);
    int t0 = a0 ? -1 : -2, t1 = a1 ? -1 : -2;
    for (int step = 0; step < 24 && (t0 == -1 || t1 == -1); ++step) {
        if (t0 == -1) t0 = table_try(vs, w0);
        if (t1 == -1) t1 = table_try(vs, w1);
    }
    *r0 = a0 ? (t0 < 0 ? 2 : t0) : -1;
    *r1 = a1 ? (t1 < 0 ? 2 : t1) : -1;
}

// test_and_set for two ids per lane; all the ids of the warp are distinct.
__device__ __forceinline__ void visited_test_and_set2(Visited& vs, uint32_t v0, bool a0, uint32_t v1, bool a1,
                                                      bool* new0, bool* new1) {
    const int lane = lane_id();
    int t0 = a0 ? 2 : -1, t1 = a1 ? 2 : -1;
    if (vs.tbits) table_test_insert2(vs, v0, a0, v1, a1, &t0, &t1);
    bool n0 = t0 == 0, n1 = t1 == 0;
    bool in0 = false, in1 = false;
    if (t0 == 2) {
        const uint32_t mask = 1u << (v0 & 31);
        n0 = !(atomicOr(vs.bits + (v0 >> 5), mask) & mask);
        in0 = n0;
    }
    if (t1 == 2) {
        const uint32_t mask = 1u << (v1 & 31);
        n1 = !(atomicOr(vs.bits + (v1 >> 5), mask) & mask);
        in1 = n1;
    }
    const uint32_t b0 = __ballot_sync(kFull, in0), b1 = __ballot_sync(kFull, in1);
    if (b0 | b1) {
        const uint32_t lt = (1u << lane) - 1u;
        const uint32_t pos0 = vs.list_n + __popc(b0 & lt);
        const uint32_t pos1 = vs.list_n + __popc(b0) + __popc(b1 & lt);
        if (in0 && pos0 < vs.list_cap) vs.list[pos0] = v0;
        if (in1 && pos1 < vs.list_cap) vs.list[pos1] = v1;
        const uint32_t total = vs.list_n + __popc(b0) + __popc(b1);
        if (total > vs.list_cap) vs.list_overflow = true;
        vs.list_n = min(total, vs.list_cap);
        vs.global_used = true;
    }
    __syncwarp();
    *new0 = n0;
    *new1 = n1;
}

__device__ __forceinline__ void table_reset(const Visited& vs) {
    if (vs.tbits) {
        // Two buckets per 16-byte store.
        uint4* t4 = reinterpret_cast<uint4*>(vs.tab);
        const uint32_t n = 1u << (vs.tbits - 1);
        for (uint32_t i = lane_id(); i < n; i += 32) t4[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
    }
}

__device__ inline void visited_clear(Visited& vs) {
    const int lane = lane_id();
    __syncwarp();
    table_reset(vs);
    if (vs.global_used) {
        if (vs.list_overflow) {
            uint4* w4 = reinterpret_cast<uint4*>(vs.bits);
            const uint64_t n4 = vs.words / 4;
            for (uint64_t i = lane; i < n4; i += 32) w4[i] = make_uint4(0, 0, 0, 0);
        } else {
            for (uint32_t i = lane; i < vs.list_n; i += 32) vs.bits[vs.list[i] >> 5] = 0u;
        }
        vs.spills++;
    }
    vs.list_n = 0;
    vs.global_used = false;
    vs.list_overflow = false;
    __threadfence_block();
    __syncwarp();
}

// Collect the not-yet-visited ids of row[start, len) (CSR order, first
// occurrence wins, marking them visited) into cvid[0, *cnt), at most
// kCandBatch of them; *consumed reports how far it got. The ids of row[0, 32)
// and row[32, 64) may be passed in preloaded (ids0/ids1, one per lane).
__device__ __forceinline__ void collect_unvisited(const DeviceGraph& g, Visited& vs, const uint32_t* __restrict__ row,
                                                  uint32_t len, uint32_t start, uint32_t* cvid, uint32_t* cnt,
                                                  uint32_t* consumed, int* error, uint32_t ids0, uint32_t ids1,
                                                  bool have_ids) {
    const int lane = lane_id();
    uint32_t c = 0;
    uint32_t i = start;
    while (i < len && c + 32 <= kCandBatch) {
        const uint32_t idx = i + lane;
        const bool act = idx < len;
        uint32_t vid = 0xffffffffu;
        if (act) vid = (have_ids && i == 0) ? ids0 : (have_ids && i == 32) ? ids1 : __ldg(row + idx);
        if (act && vid >= g.n) set_error(error, kErrBadVid);
        const uint32_t peers = __match_any_sync(kFull, vid);
        const bool first = act && ((peers & ((1u << lane) - 1u)) == 0) && vid < g.n;
        const bool is_new = visited_test_and_set(vs, vid, first);
        const uint32_t b = __ballot_sync(kFull, is_new);
        if (is_new) cvid[c + __popc(b & ((1u << lane) - 1u))] = vid;
        c += __popc(b);
        i += 32;
    }
    __syncwarp();
    *cnt = c;
    *consumed = min(i, len);
}

// collect_unvisited for a whole level-0 row of at most 64 distinct ids,
// preloaded as row[lane] (ids0) and row[32 + lane] (ids1), 0xffffffff past
// len: one pass, two ids per lane. Ids are distinct, so the order in which
// lanes insert them cannot change which are new; the new ones are written to
// cvid in row order. Returns their count.
__device__ __forceinline__ uint32_t collect_row64_unique(const DeviceGraph& g, Visited& vs, uint32_t ids0,
                                                         uint32_t ids1, uint32_t len, uint32_t* cvid, int* error) {
    const int lane = lane_id();
    const bool in0 = static_cast<uint32_t>(lane) < len, in1 = static_cast<uint32_t>(lane) + 32u < len;
    if ((in0 && ids0 >= g.n) || (in1 && ids1 >= g.n)) set_error(error, kErrBadVid);
    bool n0, n1;
    visited_test_and_set2(vs, ids0, in0 && ids0 < g.n, ids1, in1 && ids1 < g.n, &n0, &n1);
    const uint32_t b0 = __ballot_sync(kFull, n0), b1 = __ballot_sync(kFull, n1);
    const uint32_t lt = (1u << lane) - 1u;
    if (n0) cvid[__popc(b0 & lt)] = ids0;
    if (n1) cvid[__popc(b0) + __popc(b1 & lt)] = ids1;
    __syncwarp();
    return __popc(b0) + __popc(b1);
}

// ---------------------------------------------------------------------------
// Candidate queue (subsystem b). Sorted ascending by (dist, vid) in shared
// memory, one 8-byte entry {vid word, dist bits} per candidate, so a search
// step, a move or a pop test is one load; bit 31 of the vid word marks
// "explored". T = the first min(n, L)
// entries. Entries past L that tie the worst distance lb are entries the
// reference evicted from its top-L heap but still holds in its unexplored
// heap; they stay expandable until lb drops. Any entry worse than lb is dead
// and trimmed. At most L entries can tie lb, so 2L slots always suffice.
// ---------------------------------------------------------------------------
struct Queue {
    uint2* e;        // entries {vid word, dist bits}: one 8-byte access per entry
    uint32_t n;
    uint32_t L;
    uint32_t cap;
    uint32_t hint;   // no unexplored entry before this index
    float lb;        // d[L-1] once n >= L
};

__device__ __forceinline__ float ent_d(uint2 w) { return __uint_as_float(w.y); }
__device__ __forceinline__ uint2 make_ent(float d, uint32_t v) { return make_uint2(v, __float_as_uint(d)); }

__device__ __forceinline__ uint32_t queue_lower_bound(const Queue& q, float d, uint32_t v) {
    const int lane = lane_id();
    uint32_t lo = 0, hi = q.n;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        bool less = false;
        if (idx < hi) {
            const uint2 w = q.e[idx];
            less = entry_less(ent_d(w), w.x, d, v);
        }
        const int c = __popc(__ballot_sync(kFull, less));
        const uint32_t new_lo = c == 0 ? lo : lo + (c - 1) * step + 1;
        const uint32_t new_hi = min(hi, lo + c * step);
        lo = new_lo;
        hi = new_hi;
    }
    const uint32_t idx = lo + lane;
    bool less = false;
    if (idx < hi) {
        const uint2 w = q.e[idx];
        less = entry_less(ent_d(w), w.x, d, v);
    }
    return lo + __popc(__ballot_sync(kFull, less));
}

// Insert (d, v); the caller has already applied try_push's rejection test.
__device__ __forceinline__ bool queue_insert(Queue& q, float d, uint32_t v, int* error) {
    const int lane = lane_id();
    if (q.n >= q.cap) {
        set_error(error, kErrQueue);
        return false;
    }
    const uint32_t pos = queue_lower_bound(q, d, v);
    for (int end = static_cast<int>(q.n); end > static_cast<int>(pos); end -= 32) {
        const int s = max(static_cast<int>(pos), end - 32);
        const int idx = s + lane;
        const bool act = idx < end;
        uint2 ww = make_uint2(0u, 0u);
        if (act) ww = q.e[idx];
        __syncwarp();
        if (act) q.e[idx + 1] = ww;
        __syncwarp();
    }
    if (lane == 0) q.e[pos] = make_ent(d, v & kVidMask);
    __syncwarp();
    q.n++;
    if (pos < q.hint) q.hint = pos;
    if (q.n >= q.L) {
        q.lb = ent_d(q.e[q.L - 1]);
        if (q.n > q.L) {
            uint32_t newn = q.n;
            for (uint32_t base = q.L; base < q.n; base += 32) {
                const uint32_t idx = base + lane;
                const bool dead = idx < q.n && ent_d(q.e[idx]) > q.lb;
                const uint32_t b = __ballot_sync(kFull, dead);
                if (b) { newn = base + __ffs(b) - 1; break; }
            }
            q.n = newn;
        }
    }
    return true;
}

// First unexplored entry at or after `from`, or -1.
__device__ __forceinline__ int queue_find_unexplored(const Queue& q, uint32_t from) {
    const int lane = lane_id();
    for (uint32_t base = from; base < q.n; base += 32) {
        const uint32_t idx = base + lane;
        const bool un = idx < q.n && !(q.e[idx].x & kExplored);
        const uint32_t b = __ballot_sync(kFull, un);
        if (b) return static_cast<int>(base + __ffs(b) - 1);
    }
    return -1;
}

// pop_best_unexplored_entry + should_terminate (std_candidate_queue.hpp:398-406,
// 503-513): the first unexplored entry in order, or -1 when the reference's
// unexplored heap holds nothing at distance <= lb.
__device__ __forceinline__ int queue_pop(Queue& q) {
    const int p = queue_find_unexplored(q, q.hint);
    if (p < 0) {
        q.hint = q.n;
        return -1;
    }
    if (lane_id() == 0) q.e[p].x |= kExplored;
    __syncwarp();
    q.hint = static_cast<uint32_t>(p) + 1;
    return p;
}

// pop_best_unexplored_entry, plus a peek at the entry that would come next if
// nothing better is inserted meanwhile (-1 when none), in one scan.
__device__ __forceinline__ int queue_pop_peek(Queue& q, int* next) {
    const int lane = lane_id();
    int first = -1;
    *next = -1;
    uint32_t base = q.hint;
    for (; base < q.n; base += 32) {
        const uint32_t idx = base + lane;
        const bool un = idx < q.n && !(q.e[idx].x & kExplored);
        uint32_t b = __ballot_sync(kFull, un);
        if (b) {
            if (first < 0) {
                first = static_cast<int>(base + __ffs(b) - 1);
                b &= b - 1;
            }
            if (b) {
                *next = static_cast<int>(base + __ffs(b) - 1);
                break;
            }
        }
    }
    if (first < 0) {
        q.hint = q.n;
        return -1;
    }
    if (lane == 0) q.e[first].x |= kExplored;
    __syncwarp();
    q.hint = static_cast<uint32_t>(first) + 1;
    return first;
}

// try_push for a whole batch at once (std_candidate_queue.hpp:358-388), in
// two steps: queue_accept decides which candidates the sequential pushes
// would accept, queue_merge applies them.
// Sequentially, candidate j is rejected iff T already holds L entries at
// distance <= d_j. A rejected candidate never enters T, and every later
// candidate at a distance >= a rejected one is rejected too, so candidate j
// is accepted iff
//     #{e in T : e.dist <= d_j} + #{i < j : d_i <= d_j}  <  L,
// which every lane evaluates independently. The accepted candidates are then
// merged into the sorted array in one pass; trimming the result at the new
// lb yields exactly the state the sequential pushes leave (entries trimmed
// in between are worse than every later lb).
//
// queue_accept writes the accepted candidates (m <= cnt <= kCandBatch), in
// candidate order, to bd/bv and returns m.
__device__ inline uint32_t queue_accept(const Queue& q, const uint32_t* cvid, const float* cdist, uint32_t cnt,
                                        float* bd, uint32_t* bv) {
    const int lane = lane_id();
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t tn = min(q.n, q.L);
    // Only candidates closer than lb can enter a full T, and the earlier
    // candidates a closer one must be counted against are closer as well:
    // pre_j only involves "improving" candidates. Late in a search most
    // batches have none.
    const float lim = q.n >= q.L ? q.lb : INFINITY;
    uint32_t m = 0;
    uint32_t improving_before = 0;   // improving candidates in earlier chunks
    for (uint32_t base = 0; base < cnt; base += 32) {
        const uint32_t j = base + lane;
        const bool valid = j < cnt;
        const float d = valid ? cdist[j] : INFINITY;
        const uint32_t v = valid ? cvid[j] : 0u;
        const bool improving = valid && d < lim;
        uint32_t imask = __ballot_sync(kFull, improving);
        if (imask == 0 && improving_before == 0) continue;
        // #{e in T : e.dist <= d} < L - pre  <=>  T[L-pre-1].dist > d (or T is
        // shorter than L-pre). pre = #{i < j : d_i <= d_j} is at most ub, the
        // number of earlier improving candidates, and the test is monotone in
        // pre: a lane accepted with ub is accepted, and only lanes it leaves
        // undecided need the exact count.
        const uint32_t ub = improving_before + __popc(imask & lt_mask);
        bool acc = false;
        if (improving && ub < q.L) {
            const uint32_t idx = q.L - ub - 1;
            acc = idx >= tn || ent_d(q.e[idx]) > d;
        }
        const bool undecided = improving && !acc && ub != 0;
        if (__any_sync(kFull, undecided)) {
            // Exact pre: earlier chunks from shared memory, this chunk by
            // shuffles over the improving lanes only.
            uint32_t pre = 0;
            if (improving_before) {
                for (uint32_t i = 0; i < base; ++i) pre += cdist[i] <= d ? 1u : 0u;
            }
            for (uint32_t bits = imask & lt_mask; __any_sync(kFull, bits != 0);) {
                // each lane walks its own set of earlier improving lanes; shuffles
                // need every lane, so lanes take turns through a uniform loop.
                const int k = bits ? __ffs(bits) - 1 : 0;
                const float dk = __shfl_sync(kFull, d, k);
                if (bits) {
                    pre += dk <= d ? 1u : 0u;
                    bits &= bits - 1;
                }
            }
            if (undecided && pre < q.L) {
                const uint32_t idx = q.L - pre - 1;
                acc = idx >= tn || ent_d(q.e[idx]) > d;
            }
        }
        const uint32_t b = __ballot_sync(kFull, acc);
        if (acc) {
            const uint32_t k = m + __popc(b & lt_mask);
            bd[k] = d;
            bv[k] = v;
        }
        m += __popc(b);
        improving_before += __popc(imask);
    }
    __syncwarp();
    return m;
}

// Number of entries of the sorted array q[0, n) before (d, v) by (dist, vid).
__device__ __forceinline__ uint32_t old_lower_bound(const Queue& q, float d, uint32_t v) {
    uint32_t lo = 0, hi = q.n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint2 w = q.e[mid];
        if (entry_less(ent_d(w), w.x, d, v)) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Merges the m (<= kCandBatch) accepted entries of bd/bv into the sorted
// array and trims it at the new lb. The batch is first sorted by (dist, vid)
// in place (each lane holds at most two entries in registers). A vid word may
// carry the explored bit (an entry popped before it is merged); ordering
// ignores it.
// Returns true when an entry that may still be live was dropped: with a
// capacity below 2L (the compact layout), entries past the capacity are not
// kept; they are dead unless every kept entry past L ties lb, which is what
// is reported (the caller then hands the query to the full-capacity rerun).
__device__ inline bool queue_merge(Queue& q, float* bd, uint32_t* bv, uint32_t m) {
    const int lane = lane_id();
    if (m == 0) return false;
    const bool truncated = q.n + m > q.cap;
    {
        float sd[2];
        uint32_t sv[2], rk[2];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const uint32_t k = lane + 32u * t;
            rk[t] = 0xffffffffu;
            if (k < m) {
                sd[t] = bd[k];
                sv[t] = bv[k];
                uint32_t r = 0;
                for (uint32_t i = 0; i < m; ++i) r += entry_less(bd[i], bv[i], sd[t], sv[t]) ? 1u : 0u;
                rk[t] = r;
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            if (rk[t] != 0xffffffffu) {
                bd[rk[t]] = sd[t];
                bv[rk[t]] = sv[t];
            }
        }
        __syncwarp();
    }
    // Final positions of the batch entries: rank in the old array + rank in
    // the batch (sorted, distinct); lanes past m hold a sentinel above every
    // position.
    constexpr int kNoPos = 0x7fffffff;
    int posb0 = kNoPos, posb1 = kNoPos;
    if (static_cast<uint32_t>(lane) < m) posb0 = static_cast<int>(old_lower_bound(q, bd[lane], bv[lane]) + lane);
    const bool two = m > 32u;
    if (two && static_cast<uint32_t>(lane) + 32u < m)
        posb1 = static_cast<int>(old_lower_bound(q, bd[lane + 32], bv[lane + 32]) + lane + 32u);
    const int p0 = __shfl_sync(kFull, posb0, 0);   // position of the smallest batch entry
    // Output positions [p0, end) change. Output o holds batch entry r when
    // o = posb_r, else the old entry o - #{r : posb_r < o}, which lies at or
    // before o; within a chunk of 32 outputs every lane reads its source
    // before any lane writes. Chunks go tail first: a chunk's sources lie
    // before the outputs of every chunk written earlier.
    const int end = static_cast<int>(min(q.n + m, q.cap));
    const uint32_t lt = (1u << lane) - 1u;
    for (int cb = end - 32; cb + 32 > p0; cb -= 32) {
        const uint32_t rel0 = static_cast<uint32_t>(posb0) - static_cast<uint32_t>(cb);
        const uint32_t rel1 = static_cast<uint32_t>(posb1) - static_cast<uint32_t>(cb);
        uint32_t mask = __reduce_or_sync(kFull, rel0 < 32u ? 1u << rel0 : 0u);   // batch outputs in the chunk
        uint32_t nb = __popc(__ballot_sync(kFull, posb0 < cb));                 // batch outputs before it
        if (two) {
            mask |= __reduce_or_sync(kFull, rel1 < 32u ? 1u << rel1 : 0u);
            nb += __popc(__ballot_sync(kFull, posb1 < cb));
        }
        const int before = static_cast<int>(nb + __popc(mask & lt));
        const int o = cb + lane;
        const bool act = o >= p0;
        const bool from_batch = (mask >> lane) & 1u;
        uint2 ww = make_uint2(0u, 0u);
        if (act) ww = from_batch ? make_ent(bd[before], bv[before]) : q.e[o - before];
        __syncwarp();
        if (act) q.e[o] = ww;
    }
    __syncwarp();
    const uint32_t total = min(q.n + m, q.cap);
    q.n = total;
    if (static_cast<uint32_t>(p0) < q.hint) q.hint = static_cast<uint32_t>(p0);
    if (q.n >= q.L) {
        q.lb = ent_d(q.e[q.L - 1]);
        uint32_t newn = q.n;
        for (uint32_t base = q.L; base < q.n; base += 32) {
            const uint32_t idx = base + lane;
            const bool dead = idx < q.n && ent_d(q.e[idx]) > q.lb;
            const uint32_t b = __ballot_sync(kFull, dead);
            if (b) { newn = base + __ffs(b) - 1; break; }
        }
        q.n = newn;
    }
    return truncated && q.n == q.cap;
}

// try_push of a whole batch (bd/bv: scratch for the accepted entries).
__device__ inline bool queue_push_batch(Queue& q, uint32_t* cvid, float* cdist, uint32_t cnt, float* bd, uint32_t* bv,
                                        int* error) {
    (void)error;
    return queue_merge(q, bd, bv, queue_accept(q, cvid, cdist, cnt, bd, bv));
}

// The smallest accepted entry of bd/bv[0, m) by (dist, vid), m >= 1: its index
// (in every lane), distance and vid word.
__device__ __forceinline__ uint32_t batch_argmin(const float* bd, const uint32_t* bv, uint32_t m, float* d_out,
                                                 uint32_t* v_out) {
    const int lane = lane_id();
    float md = INFINITY;
    uint32_t mv = 0xffffffffu, mi = 0xffffffffu;
    for (uint32_t k = lane; k < m; k += 32) {
        const float d = bd[k];
        const uint32_t v = bv[k];
        if (mi == 0xffffffffu || entry_less(d, v, md, mv)) { md = d; mv = v; mi = k; }
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float od = __shfl_xor_sync(kFull, md, off);
        const uint32_t ov = __shfl_xor_sync(kFull, mv, off);
        const uint32_t oi = __shfl_xor_sync(kFull, mi, off);
        if (oi != 0xffffffffu && (mi == 0xffffffffu || entry_less(od, ov, md, mv))) { md = od; mv = ov; mi = oi; }
    }
    *d_out = md;
    *v_out = mv;
    return mi;
}

// ---------------------------------------------------------------------------
// Row lookup: fetch_level_nbrs (index/compact_structure/hierarchical_graph.hpp:99-108).
// ---------------------------------------------------------------------------
__device__ __forceinline__ const uint32_t* level_row(const DeviceGraph& g, uint32_t vid, uint32_t level,
                                                     uint32_t* len) {
    const uint2 info = __ldg(g.vinfo + vid);
    const uint32_t hl = info.x;
    if (hl == kInvalidLevel || hl < level || hl >= kMaxGroups) {
        *len = 0;
        return g.nbrs;
    }
    const uint64_t row = static_cast<uint64_t>(info.y) * (hl + 1ull) + (hl - level);
    const uint64_t* off = g.offsets[hl];
    const uint64_t b = __ldg(reinterpret_cast<const unsigned long long*>(off + row));
    const uint64_t e = __ldg(reinterpret_cast<const unsigned long long*>(off + row + 1));
    *len = static_cast<uint32_t>(e - b);
    return g.nbrs + b;
}

struct Counters {
    uint32_t dist_evals, upper_rows, upper_row_ids, l0_rows, l0_row_ids, upper_dist_evals;
};

// Accumulates clock64() deltas per phase when enabled (warp-uniform flag);
// the accumulators live in the warp's shared memory, lane 0 updates them.
struct PhaseClock {
    bool on;
    long long t;
    unsigned long long* acc;
    __device__ __forceinline__ void start(bool enabled, unsigned long long* smem_acc) {
        on = enabled;
        acc = smem_acc;
        if (on) {
            if (lane_id() < kPhases) acc[lane_id()] = 0;
            __syncwarp();
            t = clock64();
        }
    }
    __device__ __forceinline__ void lap(int phase) {
        if (on) {
            const long long now = clock64();
            if (lane_id() == 0) acc[phase] += static_cast<unsigned long long>(now - t);
            t = now;
        }
    }
    __device__ __forceinline__ void count(int phase) {
        if (on && lane_id() == 0) acc[phase] += 1;
    }
};

// Shared memory words per warp for a launch.
constexpr uint32_t kPhaseWords = 2 * kPhases;   // kPhases uint64 accumulators

// Staged rows: a 4-word mbarrier slot, then kStageRows rows of dim + kStagePad words.
__host__ __device__ inline uint32_t stage_words(uint32_t dim, uint32_t stage_rows) {
    return stage_rows ? 4u + stage_rows * (dim + kStagePad) : 0u;
}

// The queue's entry array holds an even number of 8-byte entries
// (2 * queue_words(cap) words), so that the regions after it (the visited
// table, read 16 bytes at a time when cleared, the next warp's area) stay
// 16-byte aligned whatever the capacity (dim, the stage and the fixed parts
// are multiples of 4 words).
__host__ __device__ inline uint32_t queue_words(uint32_t cap) { return (cap + 1u) & ~1u; }

__host__ __device__ inline uint32_t warp_smem_words(uint32_t dim, uint32_t cap, uint32_t vh_bits,
                                                    uint32_t stage_rows = 0) {
    return dim + 2 * queue_words(cap) + 4 * kCandBatch + (vh_bits ? 4u * (1u << vh_bits) : 0u) + kPhaseWords +
           stage_words(dim, stage_rows);
}

struct WarpSmem {
    unsigned long long* phase;   // kPhases accumulators (8-byte aligned: first)
    unsigned long long* mbar;    // staging mbarrier (null without staging)
    float* stage;                // staged rows, 16-byte aligned (null without staging)
    float* q;
    uint2* qe;
    uint32_t* cvid;
    float* cdist;
    float* bd;
    uint32_t* bv;
    uint32_t* vh;
    CoopCtl* coop;               // cooperative search's control block (null otherwise)
};

__device__ __forceinline__ WarpSmem carve(float* base, uint32_t dim, uint32_t cap, uint32_t stage_rows = 0) {
    WarpSmem s;
    s.phase = reinterpret_cast<unsigned long long*>(base);
    s.mbar = stage_rows ? reinterpret_cast<unsigned long long*>(base + kPhaseWords) : nullptr;
    s.stage = stage_rows ? base + kPhaseWords + 4 : nullptr;
    s.q = base + kPhaseWords + stage_words(dim, stage_rows);
    s.qe = reinterpret_cast<uint2*>(s.q + dim);
    s.cvid = reinterpret_cast<uint32_t*>(s.q + dim + 2 * queue_words(cap));
    s.cdist = reinterpret_cast<float*>(s.cvid + kCandBatch);
    s.bd = s.cdist + kCandBatch;
    s.bv = reinterpret_cast<uint32_t*>(s.bd + kCandBatch);
    s.vh = s.bv + kCandBatch;
    s.coop = nullptr;
    return s;
}

// ---------------------------------------------------------------------------
// Level-0 beam search, pipelined across expansions (single_layer_router.hpp:
// 145-163, beam_loop.hpp:90-119), for graphs whose level-0 rows hold at most 64
// distinct ids. On entry the queue holds the cursor and the cursor is visited.
//
// The reference pops the next entry only after pushing every candidate of the
// current row. That entry is known earlier: once the current batch's
// acceptance is decided, the next pop is the smaller (by dist, vid) of
//   * p2, the first unexplored entry after the one being expanded, and
//   * the smallest accepted candidate of the batch,
// because every other unexplored entry is larger than p2, rejected candidates
// never enter the unexplored heap, and the smallest accepted candidate always
// ends inside the top L (all entries before it are old entries, fewer than L
// by its acceptance). p2 cannot be trimmed by the merge either: if it is the
// smaller, it is at most the smallest accepted candidate, which stays within
// lb. With neither, should_terminate holds (std_candidate_queue.hpp:503-513).
// So the next expansion's row is collected (visited test_and_set; the merge
// does not touch the visited set) and its first rows' loads are issued before
// the current batch is merged, and the merge runs while they are in flight.
// The chosen entry is marked explored where it lies: p2 in the array, a new
// candidate in the batch before the merge places it.
// ---------------------------------------------------------------------------
// Returns true when the compact queue lost a live entry (see queue_merge).
template <int kMetric, bool kExact, bool kRegs>
__device__ __forceinline__ bool l0_search_pipelined(const SearchArgs& a, Queue& q, Visited& vs, const WarpSmem& sm,
                                                    float qsq, uint32_t cur, Counters& ct, PhaseClock& pc,
                                                    Stage& st) {
    const int lane = lane_id();
    const DeviceGraph& g = a.g;
    const bool l2_next = a.pf_l2 != 0;
    uint32_t* cv = sm.cvid;
    float* cd = sm.cdist;
    // Pop the cursor: the queue's only entry.
    if (lane == 0) q.e[0].x |= kExplored;
    __syncwarp();
    q.hint = 1;
    unsigned long long desc = __ldg(g.l0row + cur);
    uint32_t len = static_cast<uint32_t>(desc >> kRowLenShift);
    const uint32_t* row = g.nbrs + (desc & kRowStartMask);
    uint32_t ids0 = lane < len ? __ldg(row + lane) : 0xffffffffu;
    uint32_t ids1 = lane + 32 < len ? __ldg(row + lane + 32) : 0xffffffffu;
    uint32_t cnt = collect_row64_unique(g, vs, ids0, ids1, len, cv, a.error);
    ct.l0_rows++;
    ct.l0_row_ids += len;
    ulonglong2 pre[kBlock];
    dist_preload<kRegs>(g, cv, cnt, pre, l2_next);
    pc.lap(kPhCollect);
    // The predicted entry after the one being expanded: its index (-1: none),
    // vid, row descriptor and, once loaded, ids.
    int p2 = -1;
    uint32_t pf_vid = kVidMask;
    unsigned long long pf_desc = 0ull;
    uint32_t pf_ids0 = 0u, pf_ids1 = 0u;
    bool pf_have_ids = false;
    for (uint32_t it = 0;; ++it) {
        if (it > g.n) { set_error(a.error, kErrBound); break; }
        if (cnt) batch_distances<kMetric, kExact, false, kRegs>(g, sm.q, qsq, cv, cd, cnt, st, a.error, &pre);
        ct.dist_evals += cnt;
        if (p2 >= 0 && !pf_have_ids) {
            // The predicted entry's descriptor has arrived by now: fetch its ids.
            const uint32_t len2 = static_cast<uint32_t>(pf_desc >> kRowLenShift);
            const uint32_t* row2 = g.nbrs + (pf_desc & kRowStartMask);
            pf_ids0 = lane < len2 ? __ldg(row2 + lane) : 0xffffffffu;
            pf_ids1 = lane + 32 < len2 ? __ldg(row2 + lane + 32) : 0xffffffffu;
            pf_have_ids = true;
        }
        pc.lap(kPhDist);
        const uint32_t m = cnt ? queue_accept(q, cv, cd, cnt, sm.bd, sm.bv) : 0u;
        // The next pop: min(p2, smallest accepted), or termination.
        bool take_new = false;
        uint32_t next = kVidMask;
        if (m) {
            float bdm;
            uint32_t bvm;
            const uint32_t bi = batch_argmin(sm.bd, sm.bv, m, &bdm, &bvm);
            take_new = p2 < 0 || entry_less(bdm, bvm, ent_d(q.e[p2]), q.e[p2].x);
            if (take_new) {
                next = bvm & kVidMask;
                if (lane == 0) sm.bv[bi] = bvm | kExplored;
            }
        }
        if (!take_new && p2 >= 0) {
            next = q.e[p2].x & kVidMask;
            if (lane == 0) q.e[p2].x |= kExplored;
            q.hint = static_cast<uint32_t>(p2) + 1;
        }
        __syncwarp();
        // CandidateEntry::is_invalid ends the loop as the reference's pop of an
        // invalid entry does (cannot occur on validated graphs).
        const bool go = (take_new || p2 >= 0) && next != kVidMask;
        uint32_t ncnt = 0;
        if (go) {
            const bool hit = !take_new && next == pf_vid;
            if (hit) pc.count(kPhPrefetchHits);
            desc = hit ? pf_desc : __ldg(g.l0row + next);
            len = static_cast<uint32_t>(desc >> kRowLenShift);
            row = g.nbrs + (desc & kRowStartMask);
            if (hit && pf_have_ids) {
                ids0 = pf_ids0;
                ids1 = pf_ids1;
            } else {
                ids0 = lane < len ? __ldg(row + lane) : 0xffffffffu;
                ids1 = lane + 32 < len ? __ldg(row + lane + 32) : 0xffffffffu;
            }
            pf_have_ids = false;
            pc.lap(kPhPop);
            // The current candidates are in bd/bv now: cv takes the next row's.
            ncnt = collect_row64_unique(g, vs, ids0, ids1, len, cv, a.error);
            ct.l0_rows++;
            ct.l0_row_ids += len;
            dist_preload<kRegs>(g, cv, ncnt, pre, l2_next);
            pc.lap(kPhCollect);
        }
        // The current batch's merge runs while the next rows are loaded.
        const bool lost = queue_merge(q, sm.bd, sm.bv, m);
        __syncwarp();
        pc.lap(kPhMerge);
        if (lost && a.compact) return true;
        if (!go) break;
        // Predict the entry after `next`: the first unexplored entry now.
        p2 = queue_find_unexplored(q, q.hint);
        if (p2 >= 0) {
            q.hint = static_cast<uint32_t>(p2);
            pf_vid = q.e[p2].x & kVidMask;
            pf_desc = __ldg(g.l0row + pf_vid);
        } else {
            q.hint = q.n;
            pf_vid = kVidMask;
        }
        pc.lap(kPhPop);
        cnt = ncnt;
    }
    return false;
}

// ---------------------------------------------------------------------------
// One query (hierarchical_graph_router.hpp:195-248; query_l0_only :258-286).
// ---------------------------------------------------------------------------
// stage_phase: with kStage, the parity of the next phase of the warp's staging
// mbarrier, which the caller initialised once (an mbarrier is not initialised
// again while it is valid) and which carries over from query to query.
// kPipe: the kernel carries the pipelined level-0 loop (taken when a.l0_pipe;
// otherwise, and in kernels without it, one expansion at a time). kRegs: the
// pipelined loop holds the next expansion's first pass in registers (the
// 128-register budget) instead of prefetching it into L2. kW: warps per query.
// kTrace: record the search in a.tr (the probes' trace kernel).
template <int kMetric, bool kExact, bool kStage = false, bool kRegs = false, int kW = 1, bool kPipe = false,
          bool kTrace = false>
__device__ void search_one(const SearchArgs& a, uint32_t qi, uint32_t slot, const WarpSmem& sm,
                           uint32_t* stage_phase = nullptr) {
    const int lane = lane_id();
    const DeviceGraph& g = a.g;
    const uint32_t dim = g.dim;
    const uint32_t topk = a.topk ? (a.coherent ? __ldcg(a.topk + qi) : a.topk[qi]) : a.topk_default;
    const uint32_t L = a.queue ? (a.coherent ? __ldcg(a.queue + qi) : a.queue[qi]) : a.queue_default;
    uint64_t* out = a.out + static_cast<size_t>(qi) * a.k_stride;
    constexpr uint64_t kInvalidWord = (static_cast<uint64_t>(0x7f7fffffu) << 32) | kVidMask;

    if (topk > a.k_stride || L < topk || (a.compact ? L + 1ull : 2ull * L) > a.cap) {
        set_error(a.error, kErrArgs);
        for (uint32_t i = lane; i < a.k_stride; i += 32) out[i] = kInvalidWord;
        return;
    }

    Counters ct = {};
    uint32_t nres = 0;
    bool overflowed = false;
    PhaseClock pc;
    pc.start(a.phase_cycles != nullptr, sm.phase);
    const long long t_begin = pc.on ? clock64() : 0;
    Visited vs;
    vs.tab = reinterpret_cast<uint2*>(sm.vh);
    vs.tbits = a.vh_bits ? a.vh_bits + 1 : 0u;   // a.vh_bits: log2 of the table's 16-byte units
    vs.kbits = a.vk_bits;
    vs.kmask = a.vk_bits >= 32 ? 0xFFFFFFFFu : ((1u << a.vk_bits) - 1u);
    vs.bits = a.vis_bits + static_cast<size_t>(slot) * a.words_per_slot;
    vs.list = a.vis_list + static_cast<size_t>(slot) * a.list_cap;
    vs.list_n = 0;
    vs.list_cap = a.list_cap;
    vs.words = a.words_per_slot;
    vs.global_used = false;
    vs.list_overflow = false;
    vs.spills = 0;
    uint32_t* cvid = sm.cvid;
    float* cdist = sm.cdist;
    Stage st;
    st.buf = sm.stage;
    st.mbar = kStage ? smem_addr(sm.mbar) : 0u;
    st.phase = kStage ? *stage_phase : 0u;

    if (g.n != 0 && g.top != kInvalidLevel && L > 0) {
        // Stage the query row in shared memory; reset the visited hash.
        const float4* src = reinterpret_cast<const float4*>(a.queries + static_cast<size_t>(qi) * dim);
        float4* dst = reinterpret_cast<float4*>(sm.q);
        for (uint32_t i = lane; i < dim / 4; i += 32) dst[i] = a.coherent ? __ldcg(src + i) : __ldg(src + i);
        table_reset(vs);
        __syncwarp();
        const float qsq = (kMetric == ARTEA_GPU_COSINE) ? query_sqnorm<kExact>(sm.q, dim) : 0.f;

        // Entry point distance (hierarchical_graph_router.hpp:209-211).
        uint32_t cur = g.entry;
        if (lane == 0) cvid[0] = cur;
        __syncwarp();
        dist_call<kMetric, kExact, kStage, kW>(g, sm.q, qsq, cvid, cdist, 1, st, a.error, sm.coop);
        float cur_d = cdist[0];
        ct.dist_evals = 1;

        // Greedy descent, levels top..1 (hierarchical_graph_router.hpp:228-236).
        if (!a.l0_only) {
            for (uint32_t h = g.top; h >= 1; --h) {
                visited_set(vs, cur);
                for (uint32_t hop = 0;; ++hop) {
                    if (hop > g.n) { set_error(a.error, kErrBound); break; }
                    // enable_early_stop: detail/beam_loop.hpp:147-150.
                    if (a.early_stop && cur_d <= a.es_thr[h]) break;
                    uint32_t len;
                    const uint32_t* row = level_row(g, cur, h, &len);
                    ct.upper_rows++;
                    ct.upper_row_ids += len;
                    float best_d = cur_d;
                    uint32_t best_v = cur;
                    uint32_t pos = 0;
                    while (pos < len) {
                        uint32_t cnt, consumed;
                        collect_unvisited(g, vs, row, len, pos, cvid, &cnt, &consumed, a.error, 0u, 0u, false);
                        pos = consumed;
                        if (cnt == 0) continue;
                        dist_call<kMetric, kExact, kStage, kW>(g, sm.q, qsq, cvid, cdist, cnt, st, a.error,
                                                               sm.coop);
                        ct.dist_evals += cnt;
                        ct.upper_dist_evals += cnt;
                        // First strict improvement in row order (beam_loop.hpp:153-160).
                        float md = INFINITY;
                        uint32_t mi = 0xffffffffu;
                        for (uint32_t i = lane; i < cnt; i += 32) {
                            const float d = cdist[i];
                            if (d < md) { md = d; mi = i; }
                        }
                        for (int off = 16; off > 0; off >>= 1) {
                            const float od = __shfl_xor_sync(kFull, md, off);
                            const uint32_t oi = __shfl_xor_sync(kFull, mi, off);
                            if (od < md || (od == md && oi < mi)) { md = od; mi = oi; }
                        }
                        if (md < best_d) {
                            best_d = md;
                            best_v = cvid[mi];
                        }
                        __syncwarp();
                    }
                    if (best_v == cur) break;
                    cur = best_v;
                    cur_d = best_d;
                }
                visited_clear(vs);
            }
        }
        pc.lap(kPhUpper);

        // Level-0 beam search (single_layer_router.hpp:145-163, beam_loop.hpp:90-119).
        Queue q;
        q.e = sm.qe;
        q.n = 0;
        q.L = L;
        q.cap = a.cap;
        q.hint = 0;
        q.lb = FLT_MAX;
        queue_insert(q, cur_d, cur, a.error);
        visited_set(vs, cur);
        uint32_t tpos = 0, trows = 0;   // kTrace: candidates and rows recorded
        if (kTrace && lane == 0) a.tr.cur[qi] = make_uint2(cur, __float_as_uint(cur_d));
        if (kTrace && a.tr.upper_only) {
            // The greedy descent alone: level 0 is not searched.
        } else if (kPipe && !kStage && kW == 1 && a.l0_pipe) {
            overflowed = l0_search_pipelined<kMetric, kExact, kRegs>(a, q, vs, sm, qsq, cur, ct, pc, st) &&
                         a.compact;
        } else {
            // Software pipeline: while one row is processed, the row descriptor and
            // then the neighbour ids of the entry that would be expanded next are
            // already being loaded (used if that entry is indeed popped next).
            uint32_t pf_vid = cur;
            unsigned long long pf_desc = __ldg(g.l0row + cur);
            uint32_t pf_ids0 = 0u, pf_ids1 = 0u;
            bool pf_have_ids = false;
            for (uint32_t it = 0;; ++it) {
                if (it > g.n) { set_error(a.error, kErrBound); break; }
                int p2;
                const int p = queue_pop_peek(q, &p2);
                if (p < 0) break;
                const uint32_t v = q.e[p].x & kVidMask;
                if (v == kVidMask) break;   // CandidateEntry::is_invalid
                const bool hit = v == pf_vid;
                if (hit) pc.count(kPhPrefetchHits);
                const unsigned long long desc = hit ? pf_desc : __ldg(g.l0row + v);
                const uint32_t len = static_cast<uint32_t>(desc >> kRowLenShift);
                const uint32_t* row = g.nbrs + (desc & kRowStartMask);
                uint32_t ids0, ids1;
                if (hit && pf_have_ids) {
                    ids0 = pf_ids0;
                    ids1 = pf_ids1;
                } else {
                    ids0 = lane < len ? __ldg(row + lane) : 0xffffffffu;
                    ids1 = lane + 32 < len ? __ldg(row + lane + 32) : 0xffffffffu;
                }
                pf_have_ids = false;
                if (p2 >= 0) {
                    pf_vid = q.e[p2].x & kVidMask;
                    pf_desc = __ldg(g.l0row + pf_vid);
                } else {
                    pf_vid = kVidMask;
                }
                ct.l0_rows++;
                ct.l0_row_ids += len;
                pc.lap(kPhPop);
                uint32_t pos = 0;
                const bool one_pass = g.l0_unique && len <= 64u;
                while (pos < len) {
                    uint32_t cnt, consumed;
                    if (one_pass) {
                        cnt = collect_row64_unique(g, vs, ids0, ids1, len, cvid, a.error);
                        consumed = len;
                    } else {
                        collect_unvisited(g, vs, row, len, pos, cvid, &cnt, &consumed, a.error, ids0, ids1, pos == 0);
                    }
                    pos = consumed;
                    pc.lap(kPhCollect);
                    if (kTrace) {
                        if (lane == 0 && trows < a.tr.rows_cap)
                            a.tr.rows[static_cast<size_t>(qi) * a.tr.rows_cap + trows] = make_uint2(v, cnt);
                        ++trows;
                    }
                    if (cnt == 0) continue;
                    dist_call<kMetric, kExact, kStage, kW>(g, sm.q, qsq, cvid, cdist, cnt, st, a.error, sm.coop);
                    ct.dist_evals += cnt;
                    if (kTrace) {
                        for (uint32_t i = lane; i < cnt; i += 32) {
                            if (tpos + i < a.tr.cap) {
                                a.tr.ids[static_cast<size_t>(qi) * a.tr.cap + tpos + i] = cvid[i];
                                a.tr.dists[static_cast<size_t>(qi) * a.tr.cap + tpos + i] = cdist[i];
                            }
                        }
                        tpos += cnt;
                    }
                    pc.lap(kPhDist);
                    if (p2 >= 0 && !pf_have_ids) {
                        // The next entry's descriptor has arrived by now: fetch its ids
                        // while the merge runs.
                        const uint32_t len2 = static_cast<uint32_t>(pf_desc >> kRowLenShift);
                        const uint32_t* row2 = g.nbrs + (pf_desc & kRowStartMask);
                        pf_ids0 = lane < len2 ? __ldg(row2 + lane) : 0xffffffffu;
                        pf_ids1 = lane + 32 < len2 ? __ldg(row2 + lane + 32) : 0xffffffffu;
                        pf_have_ids = true;
                    }
                    overflowed = queue_push_batch(q, cvid, cdist, cnt, sm.bd, sm.bv, a.error) && a.compact;
                    __syncwarp();
                    pc.lap(kPhMerge);
                    if (overflowed) break;
                }
                if (overflowed) break;
            }
        }
        if (kTrace && lane == 0 && !a.tr.upper_only)
            a.tr.len[qi] = make_uint2(min(tpos, a.tr.cap), min(trows, a.tr.rows_cap));
        visited_clear(vs);
        if (overflowed) {
            // The compact queue could have lost a live entry: the search is
            // redone by the full-capacity rerun, which writes this row.
            if (lane == 0) {
                const uint32_t pos = atomicAdd(a.overflow, 1u);
                a.overflow[2 + pos] = qi;
            }
            __syncwarp();
            if (kStage) *stage_phase = st.phase;
            return;
        }

        // extract_results(min(topk, |T|)) (std_candidate_queue.hpp:542-561).
        const uint32_t tsize = min(q.n, q.L);
        nres = min(topk, tsize);
        for (uint32_t i = lane; i < a.k_stride; i += 32) {
            uint64_t w = kInvalidWord;
            if (i < nres) {
                const uint2 e = sm.qe[i];
                w = (static_cast<uint64_t>(e.y) << 32) | (e.x & kVidMask);
            }
            out[i] = w;
        }
    } else {
        for (uint32_t i = lane; i < a.k_stride; i += 32) out[i] = kInvalidWord;
    }

    pc.lap(kPhTail);
    if (pc.on) {
        if (lane == 0) pc.acc[kPhTotal] = static_cast<unsigned long long>(clock64() - t_begin);
        __syncwarp();
        if (lane < kPhases) a.phase_cycles[static_cast<size_t>(qi) * kPhases + lane] = pc.acc[lane];
    }
    if (a.stats && lane == 0) {
        artea_gpu_query_stats s;
        s.dist_evals = ct.dist_evals;
        s.upper_rows = ct.upper_rows;
        s.upper_row_ids = ct.upper_row_ids;
        s.l0_rows = ct.l0_rows;
        s.l0_row_ids = ct.l0_row_ids;
        s.upper_dist_evals = ct.upper_dist_evals;
        s.results = nres;
        s.visited_spills = vs.spills;
        a.stats[qi] = s;
    }
    if (kStage) *stage_phase = st.phase;
    __syncwarp();
}

// Plain schedule: one CTA of one warp per query; slot = query index
// (24 resident CTAs per SM at the 85-register budget).
template <int kMetric, bool kExact, bool kPipe>
__global__ void __launch_bounds__(32, 24) search_plain_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const uint32_t qi = blockIdx.x;
    if (qi >= a.nq) return;
    const WarpSmem sm = carve(smem, a.g.dim, a.cap);
    search_one<kMetric, kExact, false, false, 1, kPipe>(a, qi, qi, sm);
}

// Persistent schedule: warps pull query indices from a shared counter (in
// the order a.order gives, if set). kBudget sets the register budget through
// the launch bounds: 64 (4 CTAs of 256 threads per SM, 32 resident warps), 85
// (3 x 256: 80 registers used, 24 warps), 96 (5 CTAs of at most 128 threads:
// 20 warps) or 128 (4 CTAs of at most 128 threads: 16 warps; the pipelined
// level-0 loop then holds the next expansion's first rows in registers).
// (__maxnreg__ with the same counts measured slower.)
constexpr int budget_threads(int budget) { return budget >= 96 ? 128 : 256; }
constexpr int budget_min_blocks(int budget) {
    return budget == 64 ? 4 : (budget == 96 ? 5 : (budget == 128 ? 4 : 3));
}

template <int kMetric, bool kExact, int kBudget, bool kStage = false, bool kPipe = false>
__global__ void __launch_bounds__(budget_threads(kBudget), budget_min_blocks(kBudget))
    search_persistent_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + warp;
    const uint32_t stage_rows = kStage ? kStageRows : 0u;
    const WarpSmem sm = carve(smem + static_cast<size_t>(warp) * warp_smem_words(a.g.dim, a.cap, a.vh_bits,
                                                                                    stage_rows),
                              a.g.dim, a.cap, stage_rows);
    uint32_t stage_phase = 0u;
    if (kStage) {
        if (lane_id() == 0) mbar_init(smem_addr(sm.mbar));
        __syncwarp();
    }
    for (;;) {
        uint32_t qi = 0;
        if (lane_id() == 0) qi = atomicAdd(a.next_query, 1u);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= a.nq) break;
        if (a.order) qi = __ldg(a.order + qi);
        search_one<kMetric, kExact, kStage, kBudget == 128, 1, kPipe>(a, qi, slot, sm, &stage_phase);
    }
    if (kStage) {
        __syncwarp();
        if (lane_id() == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(sm.mbar)) : "memory");
    }
}

// Full-capacity rerun of the queries a compact-queue launch abandoned
// (a.overflow: count, work counter, indices). One warp per CTA, the queue at
// 2L, the HBM bitset as visited set; CTAs with nothing to do exit at once.
template <int kMetric, bool kExact>
__global__ void __launch_bounds__(32, 24) search_rerun_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const WarpSmem sm = carve(smem, a.g.dim, a.cap);
    for (;;) {
        uint32_t i = 0;
        if (lane_id() == 0) i = atomicAdd(a.overflow + 1, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= __ldcg(a.overflow)) break;
        const uint32_t qi = __ldcg(a.overflow + 2 + i);
        search_one<kMetric, kExact>(a, qi, blockIdx.x, sm);
    }
}

// Cooperative persistent schedule: a CTA of kW warps searches one query at a
// time (queries from the shared counter, in a.order if set); warp 0 runs the
// search, and every distance batch is split over the kW warps (CoopCtl).
// Launch bounds give each thread 96 registers. Rows are read with vector
// loads; the level-0 loop takes one expansion at a time.
template <int kMetric, bool kExact, int kW>
__global__ void __launch_bounds__(kW * 32, 20 / kW) search_coop_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const uint32_t words = warp_smem_words(a.g.dim, a.cap, a.vh_bits);
    WarpSmem sm = carve(smem, a.g.dim, a.cap);
    CoopCtl* coop = reinterpret_cast<CoopCtl*>(smem + words);
    sm.coop = coop;
    if (warp != 0) {
        coop_helper<kMetric, kExact, kW>(a.g, sm.q, coop, warp, a.error);
        return;
    }
    for (;;) {
        uint32_t qi = 0;
        if (lane_id() == 0) qi = atomicAdd(a.next_query, 1u);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= a.nq) break;
        if (a.order) qi = __ldg(a.order + qi);
        search_one<kMetric, kExact, false, false, kW>(a, qi, blockIdx.x, sm);
    }
    if (lane_id() == 0) coop->quit = 1u;
    coop_barrier(kW);   // the helpers see quit and leave
}

}  // namespace artea_gpu
