// Subsystem probes: each of the query path's four subsystems run on its own,
// on the memory accesses a real search makes, so that each can be measured
// alone (for example under a profiler's per-kernel counters).
//
// A trace kernel runs the search (one expansion at a time, the persistent
// schedule) and records per query the level-0 expansions, their new
// candidates and those candidates' distances (search_one with kTrace). Then:
//   (a) probe_greedy  — the search again, stopped after the upper levels;
//   (d) probe_gather  — the recorded candidates' distances, recomputed in the
//                       search's batches (rows from HBM/L2, query in shared
//                       memory), checked against the recorded ones;
//   (c) probe_visited — every recorded expansion's row read and passed
//                       through the visited set (shared-memory table + HBM
//                       bitset spills), the new-candidate counts checked;
//   (b) probe_queue   — the recorded pops and pushes replayed on the
//                       shared-memory queue, the pop order checked.
// Measurement only: there is no counterpart in the reference.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace artea_gpu {

struct ProbeArgs {
    uint32_t* counter;      // work counter (one per probe launch)
    uint32_t* mismatch;     // replays that disagreed with the trace
    uint32_t queue;         // L
    uint32_t topk;
};

constexpr int kProbeBudgetThreads = 128;

// The trace kernel: persistent, 96 registers, one expansion at a time.
template <int kMetric, bool kExact>
__global__ void __launch_bounds__(kProbeBudgetThreads, 5) probe_trace_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + warp;
    const WarpSmem sm = carve(smem + static_cast<size_t>(warp) * warp_smem_words(a.g.dim, a.cap, a.vh_bits),
                              a.g.dim, a.cap);
    for (;;) {
        uint32_t qi = 0;
        if (lane_id() == 0) qi = atomicAdd(a.next_query, 1u);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= a.nq) break;
        search_one<kMetric, kExact, false, false, 1, false, true>(a, qi, slot, sm);
    }
}

__device__ __forceinline__ uint32_t probe_next(uint32_t* counter) {
    uint32_t qi = 0;
    if (lane_id() == 0) qi = atomicAdd(counter, 1u);
    return __shfl_sync(kFull, qi, 0);
}

// (d) distance gathers: per query, the recorded batches (one per expansion).
template <int kMetric, bool kExact>
__global__ void __launch_bounds__(kProbeBudgetThreads, 5) probe_gather_kernel(SearchArgs a, ProbeArgs p) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = lane_id();
    const uint32_t dim = a.g.dim;
    float* q = smem + static_cast<size_t>(warp) * (dim + kCandBatch);
    float* cdist = q + dim;
    Stage st;
    st.buf = nullptr;
    st.mbar = 0u;
    st.phase = 0u;
    for (;;) {
        const uint32_t qi = probe_next(p.counter);
        if (qi >= a.nq) break;
        const float4* src = reinterpret_cast<const float4*>(a.queries + static_cast<size_t>(qi) * dim);
        for (uint32_t i = lane; i < dim / 4; i += 32) reinterpret_cast<float4*>(q)[i] = __ldg(src + i);
        __syncwarp();
        const float qsq = (kMetric == ARTEA_GPU_COSINE) ? query_sqnorm<kExact>(q, dim) : 0.f;
        const uint2 len = a.tr.len[qi];
        const uint32_t* ids = a.tr.ids + static_cast<size_t>(qi) * a.tr.cap;
        const float* want = a.tr.dists + static_cast<size_t>(qi) * a.tr.cap;
        const uint2* rows = a.tr.rows + static_cast<size_t>(qi) * a.tr.rows_cap;
        uint32_t off = 0, bad = 0;
        for (uint32_t r = 0; r < len.y; ++r) {
            const uint32_t cnt = rows[r].y;
            if (cnt == 0) continue;
            if (off + cnt > len.x) break;   // the trace was capped
            batch_distances<kMetric, kExact, false>(a.g, q, qsq, ids + off, cdist, cnt, st, a.error);
            for (uint32_t i = lane; i < cnt; i += 32)
                bad += __float_as_uint(cdist[i]) != __float_as_uint(want[off + i]) ? 1u : 0u;
            __syncwarp();
            off += cnt;
        }
        const uint32_t tot = __reduce_add_sync(kFull, bad);
        if (lane == 0 && tot) atomicAdd(p.mismatch, tot);
    }
}

// (c) visited set: per query, the cursor set, then every recorded
// expansion's row read and tested, then the clear.
__global__ void __launch_bounds__(kProbeBudgetThreads, 5) probe_visited_kernel(SearchArgs a, ProbeArgs p) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + warp;
    const uint32_t table_words = a.vh_bits ? 4u * (1u << a.vh_bits) : 0u;
    uint32_t* base = reinterpret_cast<uint32_t*>(smem) + static_cast<size_t>(warp) * (table_words + kCandBatch);
    uint32_t* cvid = base + table_words;
    Visited vs;
    vs.tab = reinterpret_cast<uint2*>(base);
    vs.tbits = a.vh_bits ? a.vh_bits + 1 : 0u;
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
    const int lane = lane_id();
    for (;;) {
        const uint32_t qi = probe_next(p.counter);
        if (qi >= a.nq) break;
        table_reset(vs);
        __syncwarp();
        visited_set(vs, a.tr.cur[qi].x);
        const uint2 len = a.tr.len[qi];
        const uint2* rows = a.tr.rows + static_cast<size_t>(qi) * a.tr.rows_cap;
        uint32_t bad = 0;
        for (uint32_t r = 0; r < len.y; ++r) {
            const uint2 rec = rows[r];
            const unsigned long long desc = __ldg(a.g.l0row + rec.x);
            const uint32_t rl = static_cast<uint32_t>(desc >> kRowLenShift);
            const uint32_t* row = a.g.nbrs + (desc & kRowStartMask);
            const uint32_t ids0 = static_cast<uint32_t>(lane) < rl ? __ldg(row + lane) : 0xffffffffu;
            const uint32_t ids1 = static_cast<uint32_t>(lane) + 32u < rl ? __ldg(row + lane + 32) : 0xffffffffu;
            const uint32_t cnt = collect_row64_unique(a.g, vs, ids0, ids1, rl, cvid, a.error);
            bad += cnt != rec.y ? 1u : 0u;
        }
        visited_clear(vs);
        if (lane == 0 && bad) atomicAdd(p.mismatch, bad);
    }
}

// (b) candidate queue: per query, the cursor inserted, then per recorded
// expansion a pop (checked against the recorded vid) and the push of its
// recorded batch; at the end the queue must report termination.
__global__ void __launch_bounds__(kProbeBudgetThreads, 5) probe_queue_kernel(SearchArgs a, ProbeArgs p) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = lane_id();
    const uint32_t qw = queue_words(a.cap);
    float* base = smem + static_cast<size_t>(warp) * (2 * qw + 4 * kCandBatch);
    Queue q;
    q.e = reinterpret_cast<uint2*>(base);
    uint32_t* cvid = reinterpret_cast<uint32_t*>(base + 2 * qw);
    float* cdist = reinterpret_cast<float*>(cvid + kCandBatch);
    float* bd = cdist + kCandBatch;
    uint32_t* bv = reinterpret_cast<uint32_t*>(bd + kCandBatch);
    for (;;) {
        const uint32_t qi = probe_next(p.counter);
        if (qi >= a.nq) break;
        q.n = 0;
        q.L = p.queue;
        q.cap = a.cap;
        q.hint = 0;
        q.lb = FLT_MAX;
        const uint2 cur = a.tr.cur[qi];
        queue_insert(q, __uint_as_float(cur.y), cur.x, a.error);
        const uint2 len = a.tr.len[qi];
        const uint32_t* ids = a.tr.ids + static_cast<size_t>(qi) * a.tr.cap;
        const float* dists = a.tr.dists + static_cast<size_t>(qi) * a.tr.cap;
        const uint2* rows = a.tr.rows + static_cast<size_t>(qi) * a.tr.rows_cap;
        uint32_t off = 0, bad = 0;
        bool capped = false;
        for (uint32_t r = 0; r < len.y; ++r) {
            int p2;
            const int pi = queue_pop_peek(q, &p2);
            const uint2 rec = rows[r];
            if (pi < 0 || (q.e[pi].x & kVidMask) != rec.x) {
                ++bad;
                break;
            }
            if (off + rec.y > len.x) {
                capped = true;
                break;
            }
            for (uint32_t i = lane; i < rec.y; i += 32) {
                cvid[i] = ids[off + i];
                cdist[i] = dists[off + i];
            }
            __syncwarp();
            if (rec.y) queue_push_batch(q, cvid, cdist, rec.y, bd, bv, a.error);
            __syncwarp();
            off += rec.y;
        }
        if (!bad && !capped) {
            int p2;
            if (queue_pop_peek(q, &p2) >= 0) ++bad;   // the search ended here
        }
        if (lane == 0 && bad) atomicAdd(p.mismatch, bad);
    }
}

template <int kMetric>
struct ProbeFns {
    static void* trace(bool exact) {
        return exact ? reinterpret_cast<void*>(probe_trace_kernel<kMetric, true>)
                     : reinterpret_cast<void*>(probe_trace_kernel<kMetric, false>);
    }
    static void* gather(bool exact) {
        return exact ? reinterpret_cast<void*>(probe_gather_kernel<kMetric, true>)
                     : reinterpret_cast<void*>(probe_gather_kernel<kMetric, false>);
    }
};

void* pick_probe(int metric, bool exact, bool gather) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR:
            return gather ? ProbeFns<ARTEA_GPU_EUCLIDEAN_SQR>::gather(exact) : ProbeFns<ARTEA_GPU_EUCLIDEAN_SQR>::trace(exact);
        case ARTEA_GPU_EUCLIDEAN:
            return gather ? ProbeFns<ARTEA_GPU_EUCLIDEAN>::gather(exact) : ProbeFns<ARTEA_GPU_EUCLIDEAN>::trace(exact);
        case ARTEA_GPU_COSINE:
            return gather ? ProbeFns<ARTEA_GPU_COSINE>::gather(exact) : ProbeFns<ARTEA_GPU_COSINE>::trace(exact);
        case ARTEA_GPU_DOT:
            return gather ? ProbeFns<ARTEA_GPU_DOT>::gather(exact) : ProbeFns<ARTEA_GPU_DOT>::trace(exact);
        default: return nullptr;
    }
}

}  // namespace artea_gpu

using namespace artea_gpu;

namespace {

struct ProbeBuffers {
    std::vector<void*> ptrs;
    ~ProbeBuffers() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int alloc(T** p, size_t n) {
        if (int rc = dev_alloc(p, n)) return rc;
        ptrs.push_back(*p);
        return ARTEA_GPU_OK;
    }
};

int launch_timed(const void* fn, uint32_t grid, uint32_t threads, uint32_t smem, void** args, cudaStream_t st,
                 float* ms) {
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    cudaEventRecord(e0, st);
    const cudaError_t le = cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, st);
    cudaEventRecord(e1, st);
    const cudaError_t se = cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string("probe launch: ") + cudaGetErrorString(le));
    if (se != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string("probe: ") + cudaGetErrorString(se));
    return ARTEA_GPU_OK;
}

}  // namespace

extern "C" int artea_gpu_subsystem_probe(const artea_gpu_index* ix, int metric, int mode, uint32_t topk,
                                         uint32_t queue_size, const float* d_queries, uint32_t nq,
                                         uint32_t visited_hash_bits, artea_gpu_probe_result* res) {
    if (!ix || !res) return fail(ARTEA_GPU_EINVAL, "null argument");
    std::memset(res, 0, sizeof(*res));
    if (metric < 0 || metric > 3) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    if (mode != ARTEA_GPU_MODE_EXACT && mode != ARTEA_GPU_MODE_FAST) return fail(ARTEA_GPU_EINVAL, "unknown mode");
    if (queue_size < topk || topk == 0) return fail(ARTEA_GPU_EINVAL, "need 0 < topk <= queue");
    if (queue_size > 4096) return fail(ARTEA_GPU_EINVAL, "probe: queue above 4096");
    if (nq == 0 || !d_queries) return fail(ARTEA_GPU_EINVAL, "probe: no queries");
    if (ix->top == kInvalidLevel || ix->n == 0) return fail(ARTEA_GPU_EINVAL, "probe: empty graph");
    if (!ix->l0_unique || ix->bl > 64u)
        return fail(ARTEA_GPU_EINVAL, "probe: needs level-0 rows of at most 64 distinct ids");
    if (visited_hash_bits > 12) return fail(ARTEA_GPU_EINVAL, "probe: visited_hash_bits above 12");
    DeviceGuard guard(ix->device);
    const bool exact = mode == ARTEA_GPU_MODE_EXACT;
    cudaStream_t st = nullptr;
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device));

    SearchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g.vecs = ix->d_vecs;
    a.g.xsq = ix->d_xsq;
    a.g.vinfo = ix->d_vinfo;
    a.g.nbrs = ix->d_nbrs;
    a.g.l0row = ix->d_l0row;
    a.g.n = ix->n;
    a.g.dim = ix->dim;
    a.g.top = ix->top;
    a.g.entry = ix->entry;
    a.g.l0_unique = ix->l0_unique;
    for (int h = 0; h < kMaxGroups; ++h) a.g.offsets[h] = ix->group_ptr[h];
    a.queries = d_queries;
    a.nq = nq;
    a.topk_default = topk;
    a.queue_default = queue_size;
    a.k_stride = topk;
    a.cap = std::max<uint32_t>(2u * queue_size, 2u);
    a.vh_bits = visited_hash_bits;
    a.vk_bits = visited_kbits(ix->n, a.vh_bits);
    if (!a.vk_bits) return fail(ARTEA_GPU_EINVAL, "probe: visited table too small for N");
    a.words_per_slot = ((static_cast<uint64_t>(ix->n) + 127) / 128) * 4;
    a.list_cap = std::max<uint32_t>(std::min<uint32_t>(ix->n, 32768), 64);

    // Launch shape of every probe: 4 warps per CTA, as many CTAs as fit.
    const uint32_t warps = 4;
    const uint32_t smem_trace = warp_smem_words(ix->dim, a.cap, a.vh_bits) * 4u * warps;
    const uint32_t smem_gather = (ix->dim + kCandBatch) * 4u * warps;
    const uint32_t smem_visited = ((a.vh_bits ? 4u * (1u << a.vh_bits) : 0u) + kCandBatch) * 4u * warps;
    const uint32_t smem_queue = (2u * queue_words(a.cap) + 4u * kCandBatch) * 4u * warps;
    if (smem_trace > 227u * 1024u || smem_queue > 227u * 1024u)
        return fail(ARTEA_GPU_EINVAL, "probe: queue too large for shared memory");
    void* f_trace = pick_probe(metric, exact, false);
    void* f_gather = pick_probe(metric, exact, true);
    void* f_visited = reinterpret_cast<void*>(probe_visited_kernel);
    void* f_queue = reinterpret_cast<void*>(probe_queue_kernel);
    if (!f_trace || !f_gather) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    const void* fns[4] = {f_trace, f_gather, f_visited, f_queue};
    const uint32_t smems[4] = {smem_trace, smem_gather, smem_visited, smem_queue};
    uint32_t grids[4];
    for (int i = 0; i < 4; ++i) {
        CUDA_TRY(cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smems[i])));
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fns[i], warps * 32, smems[i]));
        if (per_sm <= 0) return fail(ARTEA_GPU_EINVAL, "probe kernel does not fit on an SM");
        grids[i] = std::min<uint32_t>(static_cast<uint32_t>(per_sm * sms), (nq + warps - 1) / warps);
    }
    const uint32_t slots = std::max(grids[0], grids[2]) * warps;

    ProbeBuffers buf;
    uint32_t *d_counter = nullptr, *d_mismatch = nullptr, *d_ids = nullptr, *d_bits = nullptr, *d_list = nullptr;
    int* d_error = nullptr;
    float* d_dists = nullptr;
    uint2 *d_rows = nullptr, *d_cur = nullptr, *d_len = nullptr;
    uint64_t* d_out = nullptr;
    const uint32_t cap = 4096u + 24u * queue_size;
    const uint32_t rows_cap = 512u + 4u * queue_size;
    if (int rc = buf.alloc(&d_counter, 8)) return rc;
    if (int rc = buf.alloc(&d_mismatch, 8)) return rc;
    if (int rc = buf.alloc(&d_error, 1)) return rc;
    if (int rc = buf.alloc(&d_ids, static_cast<size_t>(nq) * cap)) return rc;
    if (int rc = buf.alloc(&d_dists, static_cast<size_t>(nq) * cap)) return rc;
    if (int rc = buf.alloc(&d_rows, static_cast<size_t>(nq) * rows_cap)) return rc;
    if (int rc = buf.alloc(&d_cur, nq)) return rc;
    if (int rc = buf.alloc(&d_len, nq)) return rc;
    if (int rc = buf.alloc(&d_out, static_cast<size_t>(nq) * topk)) return rc;
    if (int rc = buf.alloc(&d_bits, static_cast<size_t>(slots) * a.words_per_slot)) return rc;
    if (int rc = buf.alloc(&d_list, static_cast<size_t>(slots) * a.list_cap)) return rc;
    CUDA_TRY(cudaMemset(d_bits, 0, sizeof(uint32_t) * slots * a.words_per_slot));
    CUDA_TRY(cudaMemset(d_error, 0, sizeof(int)));
    CUDA_TRY(cudaMemset(d_mismatch, 0, 8 * sizeof(uint32_t)));
    a.out = d_out;
    a.vis_bits = d_bits;
    a.vis_list = d_list;
    a.error = d_error;
    a.tr.ids = d_ids;
    a.tr.dists = d_dists;
    a.tr.rows = d_rows;
    a.tr.cur = d_cur;
    a.tr.len = d_len;
    a.tr.cap = cap;
    a.tr.rows_cap = rows_cap;
    ProbeArgs pa;
    pa.mismatch = d_mismatch;
    pa.queue = queue_size;
    pa.topk = topk;

    // Trace (the search), then (a) the upper levels alone, then (d), (c), (b).
    float ms = 0.f;
    for (int phase = 0; phase < 5; ++phase) {
        CUDA_TRY(cudaMemset(d_counter, 0, 8 * sizeof(uint32_t)));
        a.next_query = d_counter;
        pa.counter = d_counter;
        pa.mismatch = d_mismatch + phase;
        void* args_search[] = {&a};
        void* args_probe[] = {&a, &pa};
        void* args_probe1[] = {&a, &pa};
        int rc = ARTEA_GPU_OK;
        if (phase == 0) {
            a.tr.upper_only = 0;
            rc = launch_timed(f_trace, grids[0], warps * 32, smem_trace, args_search, st, &ms);
            res->search_ms = ms;
        } else if (phase == 1) {
            // The upper levels alone: the trace kernel with level 0 skipped
            // (it records only the cursor, which is the same).
            a.tr.upper_only = 1;
            rc = launch_timed(f_trace, grids[0], warps * 32, smem_trace, args_search, st, &ms);
            a.tr.upper_only = 0;
            res->greedy_ms = ms;
        } else if (phase == 2) {
            rc = launch_timed(f_gather, grids[1], warps * 32, smem_gather, args_probe, st, &ms);
            res->gather_ms = ms;
        } else if (phase == 3) {
            rc = launch_timed(f_visited, grids[2], warps * 32, smem_visited, args_probe1, st, &ms);
            res->visited_ms = ms;
        } else {
            rc = launch_timed(f_queue, grids[3], warps * 32, smem_queue, args_probe1, st, &ms);
            res->queue_ms = ms;
        }
        if (rc) return rc;
    }
    uint32_t mism[8] = {};
    int h_err = 0;
    CUDA_TRY(cudaMemcpy(mism, d_mismatch, sizeof(mism), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&h_err, d_error, sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<uint2> lens(nq);
    CUDA_TRY(cudaMemcpy(lens.data(), d_len, sizeof(uint2) * nq, cudaMemcpyDeviceToHost));
    for (const uint2& l : lens) {
        res->candidates += l.x;
        res->expansions += l.y;
        if (l.x >= cap || l.y >= rows_cap) res->capped_queries++;
    }
    res->gather_mismatches = mism[2];
    res->visited_mismatches = mism[3];
    res->queue_mismatches = mism[4];
    if (h_err) return fail(ARTEA_GPU_EKERNEL, "probe kernel error " + std::to_string(h_err));
    return ARTEA_GPU_OK;
}
