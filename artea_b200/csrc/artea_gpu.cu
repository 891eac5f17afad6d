// C-ABI of the B200 query path: device-resident index, routers, launches.
// The kernels live in search.cuh; this file owns memory, streams, launch
// configuration, the autotuner and the host-buffer entry points.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <sys/stat.h>
#include <cstdlib>

#include "../../include/artea_gpu.h"
#include "common.h"
#include "internal.h"
#include "search.cuh"

namespace artea_gpu {

namespace {
thread_local std::string t_last_error;
}

int fail(int code, const std::string& msg) {
    t_last_error = msg;
    return code;
}

}  // namespace artea_gpu

struct LaunchShape {
    uint32_t warps_per_cta = 0;
    uint32_t ctas = 0;        // grid size (persistent)
    uint32_t slots = 0;       // visited slots needed
};

// One point of the tuning space: warps per CTA, log2 of the shared-memory
// visited hash size (0: no hash, the HBM bitset only) and register budget.
struct Tuning {
    uint32_t warps = 4;
    uint32_t vh_bits = 11;
    uint32_t regs = 0;   // 0: 85-register budget, 1: 64, 2: 96, 3: 128 (96 and 128: CTAs of at most 4 warps)
    uint32_t stage = 0;  // 0: rows read with vector loads; kStageRows: TMA-staged in shared memory
    uint32_t pf = 0;     // pipelined level-0 loop: 1 = the second pass's rows are prefetched into L2
    uint32_t pipe = 1;   // pipelined level-0 loop where the graph allows it (0: one expansion at a time)
    uint32_t wpq = 1;    // warps per query: > 1 = cooperative kernel, a CTA of wpq warps per query
    uint32_t slack = 0;  // queue layout: 0 = 2L entries per search; > 0 = compact, max queue + slack
                         // entries, a query that could lose a live entry is rerun at 2L
};

// One field per tuning component (graph keys, the launch-shape cache).
uint64_t tuning_bits(const Tuning& t) {
    return (static_cast<uint64_t>(t.slack) << 44) | (static_cast<uint64_t>(t.wpq) << 40) |
           (static_cast<uint64_t>(t.warps) << 32) |
           (static_cast<uint64_t>(t.pipe) << 29) |
           (static_cast<uint64_t>(t.pf) << 28) |
           (static_cast<uint64_t>(t.stage) << 24) | (static_cast<uint64_t>(t.vh_bits) << 8) |
           static_cast<uint64_t>(t.regs);
}

// Identity of a captured launch: the buffers, sizes and launch parameters.
struct GraphKey {
    const void* q;
    const void* out;
    const void* topk;
    const void* queue;
    const void* stats;
    const void* phase;
    const void* order;
    uint32_t nq, k_stride, l0_only, pad;
    uint64_t tuning;
    bool operator<(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) < 0; }
};

struct artea_gpu_router {
    artea_gpu_index* idx = nullptr;
    uint32_t topk = 0, queue = 0, max_queue = 0, cap = 0, max_batch = 0;
    int metric = 0, mode = 0, schedule = 0;
    uint32_t want_warps = 0, want_ctas_per_sm = 0, want_vh_bits = 0, want_regs = 0, want_stage = 0;
    uint32_t want_pipeline = 0, want_prefetch = 0, want_order = 0, want_wpq = 0, want_slack = 0;
    bool use_graphs = false;
    cudaStream_t stream = nullptr;
    int num_sms = 0;

    // Visited slots.
    uint32_t* d_vis_bits = nullptr;
    uint32_t* d_vis_list = nullptr;
    uint32_t slots = 0;
    uint64_t words_per_slot = 0;
    uint32_t list_cap = 0;

    uint32_t* d_counter = nullptr;
    int* d_error = nullptr;
    uint32_t* d_order = nullptr;   // query order of the persistent schedule (max_batch entries)
    uint32_t* d_overflow = nullptr;   // compact queues: count, rerun counter, max_batch query indices

    // Staging for host-buffer calls.
    float* d_queries = nullptr;
    uint64_t* d_out = nullptr;
    uint32_t* d_topk = nullptr;
    uint32_t* d_queue = nullptr;
    artea_gpu_query_stats* d_stats = nullptr;
    uint32_t stage_nq = 0, stage_kstride = 0;

    uint64_t launches = 0;
    unsigned long long* d_phase = nullptr;      // optional per-query phase cycles (caller-owned)
    std::map<uint64_t, Tuning> tuned;           // (dim, capacity, batch bucket, ...) -> launch parameters
    std::map<uint64_t, LaunchShape> shapes;     // (warps, hash bits) -> persistent grid
    Tuning last;                                // parameters of the last launch
    bool last_pipe = false, last_ordered = false;
    std::map<GraphKey, cudaGraphExec_t> graphs; // captured launches (use_graphs)
    bool early_stop = false;                    // artea_gpu_router_set_early_stop
    float es_thr[artea_gpu::kMaxGroups] = {};
};

namespace artea_gpu {

// x.x of every vector row, accumulated as the cosine distance accumulates it
// (4 lanes per row, lane group g owning elements 16c + 4g .. 16c + 4g + 3 of
// every chunk c, one FMA chain per element position, then the 16-lane fold
// of the exact mode), so the stored value equals the one the distance kernel
// would compute for the row (utils/simd_distance.hpp:251-274, x's norm).
__global__ void row_sqnorm_kernel(const float* __restrict__ vecs, uint32_t n, uint32_t dim, float* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gi = lane & 3u, r = lane >> 2;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 8u; base < n; base += nwarps * 8u) {
        const uint64_t row = base + r;
        const bool valid = row < n;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        if (valid) {
            const float* p = vecs + row * dim + 4u * gi;
            for (uint32_t c = 0; c < dim; c += 16) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(p + c));
                a0 = fmaf(v.x, v.x, a0);
                a1 = fmaf(v.y, v.y, a1);
                a2 = fmaf(v.z, v.z, a2);
                a3 = fmaf(v.w, v.w, a3);
            }
        }
        const float s = fold16<true>(a0, a1, a2, a3);
        if (valid && gi == 0) out[row] = s;
    }
}

// Sets *repeat when some level-0 row of at most 64 ids names an id twice; one
// warp per vertex. Rows without repeats let the search take a whole row in one
// pass (collect_row64_unique).
__global__ void l0_rows_repeat_kernel(const unsigned long long* __restrict__ l0row,
                                      const uint32_t* __restrict__ nbrs, uint32_t n, int* repeat) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const unsigned long long d = l0row[v];
        const uint32_t len = static_cast<uint32_t>(d >> kRowLenShift);
        if (len > 64u) continue;   // warp-uniform
        const uint32_t* row = nbrs + (d & kRowStartMask);
        const bool in0 = lane < len, in1 = lane + 32u < len;
        const uint32_t x0 = in0 ? row[lane] : 0xffffffffu;
        const uint32_t x1 = in1 ? row[lane + 32u] : 0xfffffffeu;
        // Every lane takes part in both matches (a short-circuit here would
        // leave lanes out of a full-mask warp intrinsic).
        const uint32_t m0 = __match_any_sync(kFull, x0);
        const uint32_t m1 = __match_any_sync(kFull, x1);
        bool dup = (in0 && __popc(m0) > 1) || (in1 && __popc(m1) > 1);
        for (uint32_t k = 0; k < 32u; ++k) {
            const uint32_t y = __shfl_sync(kFull, x0, static_cast<int>(k));
            if (in1 && k < len && y == x1) dup = true;
        }
        if (__any_sync(kFull, dup) && lane == 0) atomicOr(repeat, 1);
    }
}

// Query order for the persistent schedule: the batch's query indices sorted by
// queue size, largest first (counting sort over log2 buckets of the queue
// size; order within a bucket is arbitrary). Work stealing then starts the
// longest searches first and the short ones fill the tail. One CTA.
__global__ void __launch_bounds__(1024) order_by_queue_kernel(const uint32_t* __restrict__ queue, uint32_t nq,
                                                              uint32_t* __restrict__ order) {
    __shared__ uint32_t cnt[32];
    __shared__ uint32_t next[32];
    if (threadIdx.x < 32) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x) {
        const uint32_t L = __ldg(queue + i);
        atomicAdd(&cnt[L ? 31 - __clz(L) : 0], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        // next[b] = number of queries in the buckets above b (descending order).
        uint32_t above = 0;
        for (uint32_t c = threadIdx.x + 1; c < 32; ++c) above += cnt[c];
        next[threadIdx.x] = above;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x) {
        const uint32_t L = __ldg(queue + i);
        order[atomicAdd(&next[L ? 31 - __clz(L) : 0], 1u)] = i;
    }
}

}  // namespace artea_gpu

namespace {

using namespace artea_gpu;

// Router option visited_hash_bits: 0 = autotuned, ~0u = no hash, else log2 size.
constexpr uint32_t kNoHash = 0xffffffffu;
uint32_t hash_bits_of(uint32_t want) { return want == kNoHash ? 0u : want; }
// Router option stage_rows: 0 = autotuned, ~0u = vector loads, else staged.
uint32_t stage_of(uint32_t want) { return want == kNoHash ? 0u : kStageRows; }

using KernelFn = void (*)(SearchArgs);

// regs: 0 = 85-register budget (80 registers, 24 warps per SM), 1 = 64,
// 2 = 96 (CTAs of at most 4 warps) (persistent only); stage: rows staged in
// shared memory by TMA.
// Kernels with the pipelined level-0 loop exist for the 96- and 128-register
// budgets (the 128-register kernel always carries it; it falls back to one
// expansion at a time on graphs that do not allow it); the others run one
// expansion at a time.
template <int kMetric, bool kExact, bool kStage>
KernelFn pick_persistent_s(uint32_t regs, bool pipe) {
    switch (regs) {
        case 1: return search_persistent_kernel<kMetric, kExact, 64, kStage>;
        case 2:
            if (pipe) return kStage ? nullptr : search_persistent_kernel<kMetric, kExact, 96, false, true>;
            return search_persistent_kernel<kMetric, kExact, 96, kStage>;
        case 3: return kStage ? nullptr : search_persistent_kernel<kMetric, kExact, 128, false, true>;
        default: return search_persistent_kernel<kMetric, kExact, 85, kStage>;
    }
}

template <int kMetric, bool kExact>
KernelFn pick_persistent(uint32_t regs, bool stage, bool pipe) {
    return stage ? pick_persistent_s<kMetric, kExact, true>(regs, pipe)
                 : pick_persistent_s<kMetric, kExact, false>(regs, pipe);
}

// Router option register_budget (64, 85, 96, 128) <-> Tuning::regs (1, 0, 2, 3).
uint32_t regs_index(uint32_t budget) {
    return budget == 64 ? 1u : (budget == 96 ? 2u : (budget == 128 ? 3u : 0u));
}
uint32_t regs_budget(uint32_t index) {
    return index == 1 ? 64u : (index == 2 ? 96u : (index == 3 ? 128u : 85u));
}

template <int kMetric>
KernelFn pick_kernel_m(bool exact, bool persistent, uint32_t regs, bool stage, bool pipe) {
    if (persistent)
        return exact ? pick_persistent<kMetric, true>(regs, stage, pipe) : pick_persistent<kMetric, false>(regs, stage, pipe);
    if (pipe) return exact ? search_plain_kernel<kMetric, true, true> : search_plain_kernel<kMetric, false, true>;
    return exact ? search_plain_kernel<kMetric, true, false> : search_plain_kernel<kMetric, false, false>;
}

template <int kMetric>
KernelFn pick_coop_m(bool exact, uint32_t wpq) {
    if (wpq == 2) return exact ? search_coop_kernel<kMetric, true, 2> : search_coop_kernel<kMetric, false, 2>;
    if (wpq == 4) return exact ? search_coop_kernel<kMetric, true, 4> : search_coop_kernel<kMetric, false, 4>;
    return nullptr;
}

KernelFn pick_coop(int metric, bool exact, uint32_t wpq) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR: return pick_coop_m<ARTEA_GPU_EUCLIDEAN_SQR>(exact, wpq);
        case ARTEA_GPU_EUCLIDEAN: return pick_coop_m<ARTEA_GPU_EUCLIDEAN>(exact, wpq);
        case ARTEA_GPU_COSINE: return pick_coop_m<ARTEA_GPU_COSINE>(exact, wpq);
        case ARTEA_GPU_DOT: return pick_coop_m<ARTEA_GPU_DOT>(exact, wpq);
        default: return nullptr;
    }
}

KernelFn pick_rerun(int metric, bool exact) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR:
            return exact ? search_rerun_kernel<ARTEA_GPU_EUCLIDEAN_SQR, true> : search_rerun_kernel<ARTEA_GPU_EUCLIDEAN_SQR, false>;
        case ARTEA_GPU_EUCLIDEAN:
            return exact ? search_rerun_kernel<ARTEA_GPU_EUCLIDEAN, true> : search_rerun_kernel<ARTEA_GPU_EUCLIDEAN, false>;
        case ARTEA_GPU_COSINE:
            return exact ? search_rerun_kernel<ARTEA_GPU_COSINE, true> : search_rerun_kernel<ARTEA_GPU_COSINE, false>;
        case ARTEA_GPU_DOT:
            return exact ? search_rerun_kernel<ARTEA_GPU_DOT, true> : search_rerun_kernel<ARTEA_GPU_DOT, false>;
        default: return nullptr;
    }
}

KernelFn pick_kernel(int metric, bool exact, bool persistent, uint32_t regs = 0, bool stage = false,
                     bool pipe = false) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR: return pick_kernel_m<ARTEA_GPU_EUCLIDEAN_SQR>(exact, persistent, regs, stage, pipe);
        case ARTEA_GPU_EUCLIDEAN: return pick_kernel_m<ARTEA_GPU_EUCLIDEAN>(exact, persistent, regs, stage, pipe);
        case ARTEA_GPU_COSINE: return pick_kernel_m<ARTEA_GPU_COSINE>(exact, persistent, regs, stage, pipe);
        case ARTEA_GPU_DOT: return pick_kernel_m<ARTEA_GPU_DOT>(exact, persistent, regs, stage, pipe);
        default: return nullptr;
    }
}

uint32_t smem_bytes_per_warp(uint32_t dim, uint32_t cap, uint32_t vh_bits, uint32_t stage = 0) {
    return warp_smem_words(dim, cap, vh_bits, stage) * 4u;
}

// Captured graphs hold buffer addresses: drop them whenever a buffer moves.
void clear_graphs(artea_gpu_router* r) {
    if (!r->graphs.empty()) {
        cudaStreamSynchronize(r->stream);
        cudaDeviceSynchronize();
    }
    for (auto& kv : r->graphs) cudaGraphExecDestroy(kv.second);
    r->graphs.clear();
}

int ensure_slots(artea_gpu_router* r, uint32_t slots) {
    if (slots <= r->slots) return ARTEA_GPU_OK;
    clear_graphs(r);
    dev_free(r->d_vis_bits);
    dev_free(r->d_vis_list);
    r->slots = 0;
    const size_t words = r->words_per_slot * slots;
    if (int rc = dev_alloc(&r->d_vis_bits, words)) return rc;
    if (int rc = dev_alloc(&r->d_vis_list, static_cast<size_t>(r->list_cap) * slots)) return rc;
    CUDA_TRY(cudaMemsetAsync(r->d_vis_bits, 0, sizeof(uint32_t) * words, r->stream));
    r->slots = slots;
    return ARTEA_GPU_OK;
}

int ensure_stage(artea_gpu_router* r, uint32_t nq, uint32_t k_stride) {
    if (nq <= r->stage_nq && k_stride <= r->stage_kstride) return ARTEA_GPU_OK;
    clear_graphs(r);
    const uint32_t n2 = std::max(nq, r->stage_nq);
    const uint32_t k2 = std::max(k_stride, r->stage_kstride);
    dev_free(r->d_queries);
    dev_free(r->d_out);
    dev_free(r->d_topk);
    dev_free(r->d_queue);
    dev_free(r->d_stats);
    r->stage_nq = r->stage_kstride = 0;
    if (int rc = dev_alloc(&r->d_queries, static_cast<size_t>(n2) * r->idx->dim)) return rc;
    if (int rc = dev_alloc(&r->d_out, static_cast<size_t>(n2) * k2)) return rc;
    if (int rc = dev_alloc(&r->d_topk, n2)) return rc;
    if (int rc = dev_alloc(&r->d_queue, n2)) return rc;
    if (int rc = dev_alloc(&r->d_stats, n2)) return rc;
    r->stage_nq = n2;
    r->stage_kstride = k2;
    return ARTEA_GPU_OK;
}

// The compact queue layout's slack: entries past the largest queue that may
// hold ties of lb before a search is handed to the full-capacity rerun.
constexpr uint32_t kCompactSlack = 64;

// Queue entries per search for a tuning point: 2L, or max queue + slack.
uint32_t launch_cap(const artea_gpu_router* r, const Tuning& t) {
    return t.slack ? std::max<uint32_t>(r->max_queue + t.slack, 2u) : r->cap;
}

// Persistent grid for a tuning point: as many CTAs per SM as fit.
int persistent_shape(artea_gpu_router* r, const Tuning& t, LaunchShape* s) {
    const uint64_t key = tuning_bits(t);
    auto hit = r->shapes.find(key);
    if (hit != r->shapes.end()) {
        *s = hit->second;
        return ARTEA_GPU_OK;
    }
    if ((t.regs == 2 || t.regs == 3) && t.warps > 4)
        return fail(ARTEA_GPU_EINVAL, "register budgets 96 and 128 allow at most 4 warps per CTA");
    const bool coop = t.wpq > 1;
    KernelFn fn = coop ? pick_coop(r->metric, r->mode == ARTEA_GPU_MODE_EXACT, t.wpq)
                       : pick_kernel(r->metric, r->mode == ARTEA_GPU_MODE_EXACT, true, t.regs, t.stage != 0,
                                     t.pipe != 0);
    if (!fn)
        return fail(ARTEA_GPU_EINVAL, "no kernel for this combination (staged rows with the 128-register budget, or "
                                      "the pipelined loop with a budget below 96)");
    const uint32_t cta_threads = coop ? t.wpq * 32 : t.warps * 32;
    const uint32_t cap = launch_cap(r, t);
    const uint32_t smem = coop ? smem_bytes_per_warp(r->idx->dim, cap, t.vh_bits) + kCoopWords * 4
                               : smem_bytes_per_warp(r->idx->dim, cap, t.vh_bits, t.stage) * t.warps;
    if (smem > 227u * 1024u) return fail(ARTEA_GPU_EINVAL, "persistent CTA needs more than 227 KB shared memory");
    CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(fn),
                                                           static_cast<int>(cta_threads), smem));
    if (per_sm <= 0) return fail(ARTEA_GPU_EINVAL, "persistent kernel does not fit on an SM (queue too large?)");
    if (r->want_ctas_per_sm) per_sm = std::min<int>(per_sm, static_cast<int>(r->want_ctas_per_sm));
    s->warps_per_cta = coop ? t.wpq : t.warps;
    s->ctas = static_cast<uint32_t>(per_sm) * static_cast<uint32_t>(r->num_sms);
    s->slots = coop ? s->ctas : s->ctas * t.warps;   // one visited slot per search in flight
    r->shapes[key] = *s;
    return ARTEA_GPU_OK;
}

int fill_args(artea_gpu_router* r, SearchArgs* a, const float* d_q, uint32_t nq, const uint32_t* d_topk,
              const uint32_t* d_queue, uint32_t k_stride, uint64_t* d_out, artea_gpu_query_stats* d_stats,
              bool l0_only) {
    const artea_gpu_index* ix = r->idx;
    std::memset(a, 0, sizeof(*a));
    a->g.vecs = ix->d_vecs;
    a->g.xsq = ix->d_xsq;
    a->g.vinfo = ix->d_vinfo;
    a->g.nbrs = ix->d_nbrs;
    a->g.l0row = ix->d_l0row;
    a->g.n = ix->n;
    a->g.dim = ix->dim;
    a->g.top = ix->top;
    a->g.entry = ix->entry;
    a->g.l0_unique = ix->l0_unique;
    for (int h = 0; h < kMaxGroups; ++h) a->g.offsets[h] = ix->group_ptr[h];
    a->queries = d_q;
    a->nq = nq;
    a->topk = d_topk;
    a->queue = d_queue;
    a->topk_default = r->topk;
    a->queue_default = r->queue;
    a->k_stride = k_stride;
    a->cap = r->cap;
    a->out = d_out;
    a->stats = d_stats;
    a->vis_bits = r->d_vis_bits;
    a->vis_list = r->d_vis_list;
    a->words_per_slot = r->words_per_slot;
    a->list_cap = r->list_cap;
    a->next_query = r->d_counter;
    a->error = r->d_error;
    a->l0_only = l0_only ? 1u : 0u;
    a->phase_cycles = r->d_phase;
    a->early_stop = r->early_stop ? 1u : 0u;
    for (int h = 0; h < kMaxGroups; ++h) a->es_thr[h] = r->es_thr[h];
    // The pipelined level-0 loop takes whole rows of distinct ids, <= 64 each
    // (prepare_launch applies the launch's tuning on top).
    a->l0_pipe = (r->want_pipeline != kNoHash && ix->l0_unique && ix->bl <= 64u) ? 1u : 0u;
    return ARTEA_GPU_OK;
}

// A launch made ready: kernel, grid, shared memory and final arguments. All
// allocation (visited slots) and attribute setting happens here, so the
// enqueue step can be captured into a CUDA graph.
struct Prepared {
    KernelFn fn = nullptr;
    uint32_t grid = 0;
    uint32_t threads = 0;
    uint32_t smem = 0;
    bool persistent = false;
    bool order = false;       // run order_by_queue_kernel first (a.order is set)
    SearchArgs a;
    // Compact queues: the rerun of abandoned queries at 2L (rerun_fn null: none).
    KernelFn rerun_fn = nullptr;
    uint32_t rerun_grid = 0, rerun_smem = 0;
    SearchArgs rerun_a;
};

int prepare_launch(artea_gpu_router* r, SearchArgs a, bool persistent, const Tuning& t, Prepared* p) {
    const bool exact = r->mode == ARTEA_GPU_MODE_EXACT;
    const bool coop = persistent && t.wpq > 1;
    // The pipelined loop runs where the graph allows it, the router and the
    // tuning ask for it, and the kernel carries it (persistent: the 96- and
    // 128-register kernels with vector loads; the 128-register kernel always
    // carries it and falls back on its own).
    const bool staged = persistent && t.stage != 0;
    const bool has_pipe = !coop && !staged && (persistent ? t.regs == 2 || t.regs == 3 : true);
    a.l0_pipe = (a.l0_pipe && t.pipe && has_pipe) ? 1u : 0u;
    const bool pipe_kernel = a.l0_pipe || (persistent && !coop && t.regs == 3);
    KernelFn fn = coop ? pick_coop(r->metric, exact, t.wpq)
                       : pick_kernel(r->metric, exact, persistent, t.regs, staged, pipe_kernel);
    if (!fn) return fail(ARTEA_GPU_EINVAL, "no kernel for this metric and option combination");
    // The compact queue layout: one-warp persistent kernels only.
    const bool compact = persistent && !coop && t.slack != 0;
    a.cap = compact ? launch_cap(r, t) : r->cap;
    a.compact = compact ? 1u : 0u;
    if (compact) {
        if (!r->d_overflow) {
            if (int rc = dev_alloc(&r->d_overflow, static_cast<size_t>(r->max_batch) + 2)) return rc;
        }
        a.overflow = r->d_overflow;
    }
    a.vh_bits = t.vh_bits;
    // The 16-bit slot (0xFFFF reserved) must hold the quotient of kbits - tbits bits.
    a.vk_bits = visited_kbits(r->idx->n, a.vh_bits);
    if (!a.vk_bits) return fail(ARTEA_GPU_EINVAL, "visited table too small for N");
    p->fn = fn;
    p->persistent = persistent;
    if (coop) {
        LaunchShape s;
        if (int rc = persistent_shape(r, t, &s)) return rc;
        p->grid = std::min(s.ctas, a.nq);
        p->threads = t.wpq * 32;
        p->smem = smem_bytes_per_warp(r->idx->dim, a.cap, t.vh_bits) + kCoopWords * 4;
        if (int rc = ensure_slots(r, p->grid)) return rc;
    } else if (persistent) {
        LaunchShape s;
        if (int rc = persistent_shape(r, t, &s)) return rc;
        const uint32_t needed_ctas = (a.nq + t.warps - 1) / t.warps;
        p->grid = std::min(s.ctas, needed_ctas);
        p->threads = t.warps * 32;
        p->smem = smem_bytes_per_warp(r->idx->dim, a.cap, t.vh_bits, t.stage) * t.warps;
        if (int rc = ensure_slots(r, p->grid * t.warps)) return rc;
    } else {
        p->grid = a.nq;
        p->threads = 32;
        p->smem = smem_bytes_per_warp(r->idx->dim, a.cap, t.vh_bits);
        if (int rc = ensure_slots(r, a.nq)) return rc;
    }
    a.vis_bits = r->d_vis_bits;
    a.vis_list = r->d_vis_list;
    a.pf_l2 = t.pf;
    // Longest searches first: only with per-query queue sizes (else every
    // query has the same size) and on the persistent schedule.
    p->order = persistent && a.queue != nullptr && a.nq > 1 && r->want_order != kNoHash;
    if (p->order) {
        if (!r->d_order) {
            if (int rc = dev_alloc(&r->d_order, r->max_batch)) return rc;
        }
        a.order = r->d_order;
    }
    // The attribute is per kernel function and other launch shapes (other
    // routers, autotuner candidates) change it: set it for every launch.
    CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(p->smem)));
    p->a = a;
    if (compact) {
        // One warp per CTA, the queue at 2L, the HBM bitset as visited set;
        // slots are the main launch's (it has finished when this starts).
        SearchArgs b = a;
        b.cap = r->cap;
        b.compact = 0;
        b.vh_bits = 0;
        b.l0_pipe = 0;
        b.order = nullptr;
        p->rerun_a = b;
        p->rerun_fn = pick_rerun(r->metric, exact);
        p->rerun_grid = std::min<uint32_t>(r->slots, static_cast<uint32_t>(4 * r->num_sms));
        p->rerun_smem = smem_bytes_per_warp(r->idx->dim, r->cap, 0);
        if (!p->rerun_fn) return fail(ARTEA_GPU_EINVAL, "no rerun kernel for this metric");
        CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(p->rerun_fn),
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p->rerun_smem)));
    }
    return ARTEA_GPU_OK;
}

int enqueue(artea_gpu_router* r, const Prepared& p, cudaStream_t st) {
    if (p.persistent) CUDA_TRY(cudaMemsetAsync(r->d_counter, 0, sizeof(uint32_t), st));
    if (p.order) {
        order_by_queue_kernel<<<1, 1024, 0, st>>>(p.a.queue, p.a.nq, r->d_order);
        CUDA_TRY(cudaGetLastError());
    }
    if (p.rerun_fn) CUDA_TRY(cudaMemsetAsync(r->d_overflow, 0, 2 * sizeof(uint32_t), st));
    p.fn<<<p.grid, p.threads, p.smem, st>>>(p.a);
    CUDA_TRY(cudaGetLastError());
    if (p.rerun_fn) {
        p.rerun_fn<<<p.rerun_grid, 32, p.rerun_smem, st>>>(p.rerun_a);
        CUDA_TRY(cudaGetLastError());
    }
    return ARTEA_GPU_OK;
}

int launch_with(artea_gpu_router* r, SearchArgs a, bool persistent, const Tuning& t, cudaStream_t st) {
    if (a.nq == 0) return ARTEA_GPU_OK;
    Prepared p;
    if (int rc = prepare_launch(r, a, persistent, t, &p)) return rc;
    if (int rc = enqueue(r, p, st)) return rc;
    r->last = t;
    r->last_pipe = p.a.l0_pipe != 0;
    r->last_ordered = p.order;
    r->launches++;
    return ARTEA_GPU_OK;
}

// CUDA-graph replay: the counter reset and the launch of one (buffers,
// tuning) combination are captured once and replayed afterwards.
int launch_graph(artea_gpu_router* r, SearchArgs a, bool persistent, const Tuning& t, cudaStream_t st) {
    if (a.nq == 0) return ARTEA_GPU_OK;
    Prepared p;
    if (int rc = prepare_launch(r, a, persistent, t, &p)) return rc;
    GraphKey key;
    std::memset(&key, 0, sizeof(key));
    key.q = p.a.queries;
    key.out = p.a.out;
    key.topk = p.a.topk;
    key.queue = p.a.queue;
    key.stats = p.a.stats;
    key.phase = p.a.phase_cycles;
    key.nq = p.a.nq;
    key.k_stride = p.a.k_stride;
    key.l0_only = p.a.l0_only;
    key.order = p.a.order;
    key.tuning = tuning_bits(t) | (persistent ? 1ull << 63 : 0) | (p.a.l0_pipe ? 1ull << 62 : 0);
    auto it = r->graphs.find(key);
    if (it == r->graphs.end()) {
        cudaGraph_t graph = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(r, p, r->stream);
        const cudaError_t ec = cudaStreamEndCapture(r->stream, &graph);
        if (rc != ARTEA_GPU_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ec != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) return fail(ARTEA_GPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        it = r->graphs.emplace(key, exec).first;
    }
    CUDA_TRY(cudaGraphLaunch(it->second, st));
    r->last = t;
    r->last_pipe = p.a.l0_pipe != 0;
    r->last_ordered = p.order;
    r->launches++;
    return ARTEA_GPU_OK;
}

// Autotuner for the persistent schedule. The first call for a (dim, queue
// capacity, batch-size bucket, per-query arrays) combination times each
// candidate on that call's batch (one warm launch, then the median of three
// timed launches, on the call's stream, waiting for each) and keeps the
// fastest: warps per CTA x visited-table size x register budget first; then,
// at the best of those, rows loaded ahead (8 or 16) and TMA-staged rows (at
// the best table size). Picks are kept per router and, for routers that fix
// none of these options, in a text file (ARTEA_TUNING_CACHE; default
// $XDG_CACHE_HOME/artea_b200/tuning.txt, else ~/.cache/artea_b200/tuning.txt;
// an empty ARTEA_TUNING_CACHE turns the file off) keyed by the GPU model, SM
// count, this library's build, the metric, mode, graph size and the
// combination above, so later processes skip the timing.
const char* kBuildId = __DATE__ " " __TIME__;

std::string tuning_cache_path() {
    const char* env = std::getenv("ARTEA_TUNING_CACHE");
    if (env) return std::string(env);
    const char* xdg = std::getenv("XDG_CACHE_HOME");
    if (xdg && *xdg) return std::string(xdg) + "/artea_b200/tuning.txt";
    const char* home = std::getenv("HOME");
    if (home && *home) return std::string(home) + "/.cache/artea_b200/tuning.txt";
    return std::string();
}

std::mutex g_tuning_file_mu;

std::string tuning_file_key(const artea_gpu_router* r, uint64_t key) {
    cudaDeviceProp prop;
    std::string gpu = "gpu";
    if (cudaGetDeviceProperties(&prop, r->idx->device) == cudaSuccess) gpu = prop.name;
    else cudaGetLastError();
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s|%d|%s|m%d|x%d|n%u|k%llx|cs%u|p%u|o%u", gpu.c_str(), r->num_sms, kBuildId,
                  r->metric, r->mode, r->idx->n, static_cast<unsigned long long>(key), r->want_ctas_per_sm,
                  r->want_pipeline, r->want_order);
    std::string k(buf);
    for (char& c : k)
        if (c == ' ') c = '_';
    return k;
}

bool tuning_file_load(const std::string& path, const std::string& fkey, Tuning* t) {
    if (path.empty()) return false;
    std::lock_guard<std::mutex> lk(g_tuning_file_mu);
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[1024];
    bool found = false;
    while (std::fgets(line, sizeof(line), f)) {
        char k[600];
        unsigned w, b, rg, st, pf, pp, q, sl;
        if (std::sscanf(line, "%599s %u %u %u %u %u %u %u %u", k, &w, &b, &rg, &st, &pf, &pp, &q, &sl) == 9 &&
            fkey == k && rg <= 3 && (st == 0 || st == kStageRows) && pf <= 1 && pp <= 1 && w >= 1 && w <= 8 &&
            b <= 12 && (q == 1 || q == 2 || q == 4) && sl <= 4096) {
            t->wpq = q;
            t->slack = sl;
            t->warps = w;
            t->vh_bits = b;
            t->regs = rg;
            t->stage = st;
            t->pf = pf;
            t->pipe = pp;
            found = true;   // the last line for a key wins
        }
    }
    std::fclose(f);
    return found;
}

void tuning_file_store(const std::string& path, const std::string& fkey, const Tuning& t) {
    if (path.empty()) return;
    std::lock_guard<std::mutex> lk(g_tuning_file_mu);
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0) {
        const std::string dir = path.substr(0, slash);   // mkdir -p, one component at a time
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return;
    std::fprintf(f, "%s %u %u %u %u %u %u %u %u\n", fkey.c_str(), t.warps, t.vh_bits, t.regs, t.stage, t.pf, t.pipe,
                 t.wpq, t.slack);
    std::fclose(f);
}

uint32_t batch_bucket(uint32_t nq) {
    uint32_t b = 0;
    while (b < 31 && (1u << b) < nq) ++b;
    return b;
}

Tuning tuned(artea_gpu_router* r, const SearchArgs& a, cudaStream_t st) {
    Tuning t;
    // Whether the pipelined loop is a choice: the graph allows it and the
    // router leaves it open (pipeline 0); pipeline 1 fixes it on.
    const bool pipe_open = a.l0_pipe && r->want_pipeline == 0;
    const bool fixed_pf = r->want_prefetch != 0 || !a.l0_pipe;
    const uint32_t pf_fixed = r->want_prefetch == 16 ? 1u : 0u;
    if (r->want_wpq > 1 && r->want_vh_bits) {
        t.wpq = r->want_wpq;
        t.warps = 1;
        t.vh_bits = hash_bits_of(r->want_vh_bits);
        t.regs = 2;
        t.stage = 0;
        t.pf = 0;
        t.pipe = 0;
        return t;
    }
    const uint32_t slack_fixed = (r->want_slack == 0 || r->want_slack == kNoHash) ? 0u : r->want_slack;
    if (r->want_wpq <= 1 && r->want_warps && r->want_vh_bits && r->want_regs && r->want_stage && fixed_pf) {
        t.warps = r->want_warps;
        t.vh_bits = hash_bits_of(r->want_vh_bits);
        t.regs = regs_index(r->want_regs);
        t.stage = stage_of(r->want_stage);
        t.pf = pf_fixed;
        t.pipe = 1;
        t.slack = t.stage ? 0u : slack_fixed;
        return t;
    }
    const uint64_t key = (static_cast<uint64_t>(r->idx->dim) << 40) | (static_cast<uint64_t>(r->cap) << 16) |
                         (static_cast<uint64_t>(batch_bucket(a.nq)) << 8) | (a.queue ? 2u : 0u) |
                         (a.l0_only ? 1u : 0u);
    auto it = r->tuned.find(key);
    if (it != r->tuned.end()) return it->second;
    const bool shared = !r->want_warps && !r->want_vh_bits && !r->want_regs && !r->want_stage && !r->want_prefetch &&
                        !r->want_wpq && !r->want_slack;
    const std::string path = shared ? tuning_cache_path() : std::string();
    const std::string fkey = shared ? tuning_file_key(r, key) : std::string();
    if (shared && tuning_file_load(path, fkey, &t)) {
        r->tuned[key] = t;
        return t;
    }
    // Candidate lists: a fixed option is its own single choice.
    std::vector<uint32_t> warp_choices = {2, 4, 8}, bit_choices = {0, 8, 9, 10}, reg_choices = {0, 1, 2, 3},
                          stage_choices = {0, kStageRows}, pf_choices = {0, 1};
    if (r->want_warps) warp_choices = {r->want_warps};
    if (r->want_vh_bits) bit_choices = {hash_bits_of(r->want_vh_bits)};
    if (r->want_regs) reg_choices = {regs_index(r->want_regs)};
    if (r->want_stage) stage_choices = {stage_of(r->want_stage)};
    if (fixed_pf) pf_choices = {pf_fixed};
    std::vector<uint32_t> pipe_choices = pipe_open ? std::vector<uint32_t>{0, 1} : std::vector<uint32_t>{1};
    // Queue layout: the compact one pays where the 2L queue is a large part
    // of a warp's shared memory.
    std::vector<uint32_t> slack_choices = {0};
    if (r->want_slack == 0 && r->max_queue >= 128) slack_choices = {0, kCompactSlack};
    else if (r->want_slack != 0 && r->want_slack != kNoHash) slack_choices = {r->want_slack};
    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    float best_ms = 1e30f;
    Tuning best;
    best.warps = warp_choices[0];
    best.vh_bits = bit_choices[0];
    best.regs = reg_choices[0];
    best.stage = stage_choices[0];
    best.pf = pf_choices[0];
    best.pipe = pipe_choices.back();
    auto time_candidate = [&](const Tuning& c) {
        if (r->want_wpq && c.wpq != r->want_wpq) return;
        if (c.slack && (c.wpq > 1 || c.stage)) return;   // compact queues: one-warp kernels, vector loads
        if (c.stage && c.pf) return;           // staged rows use the one-expansion loop
        if (c.stage && c.regs == 3) return;    // no staged 128-register kernel
        if ((c.regs == 2 || c.regs == 3) && c.warps > 4) return;
        // The 128-register budget exists for the pipelined loop's preloaded
        // rows; the one-expansion loop only loses warps with it. The
        // pipelined loop is timed with the 96- and 128-register budgets.
        if (pipe_open && c.regs == 3 && !c.pipe) return;
        if (pipe_open && c.pipe && (c.regs == 0 || c.regs == 1)) return;
        LaunchShape s;
        if (persistent_shape(r, c, &s) != ARTEA_GPU_OK) {
            cudaGetLastError();
            return;
        }
        // One warm launch, then the median of three.
        bool ok = launch_with(r, a, true, c, st) == ARTEA_GPU_OK;
        for (int rep = 0; rep < 3 && ok; ++rep) {
            cudaEventRecord(ev[rep], st);
            ok = launch_with(r, a, true, c, st) == ARTEA_GPU_OK;
        }
        if (ok) cudaEventRecord(ev[3], st);
        ok = ok && cudaEventSynchronize(ev[3]) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return;
        }
        float ms[3];
        cudaEventElapsedTime(&ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&ms[1], ev[1], ev[2]);
        cudaEventElapsedTime(&ms[2], ev[2], ev[3]);
        std::sort(ms, ms + 3);
        if (ms[1] < best_ms) {
            best_ms = ms[1];
            best = c;
        }
    };
    // 1. level-0 loop, launch shape, table size and register budget, with
    // vector loads.
    for (uint32_t slack : slack_choices)
        for (uint32_t pipe : pipe_choices)
            for (uint32_t reg : reg_choices)
                for (uint32_t w : warp_choices)
                    for (uint32_t b : bit_choices) {
                        Tuning c;
                        c.warps = w;
                        c.vh_bits = b;
                        c.regs = reg;
                        c.stage = stage_choices[0];
                        c.pf = pf_choices[0];
                        c.pipe = pipe;
                        c.slack = slack;
                        time_candidate(c);
                    }
    // 1b. warps per query: the cooperative kernel (96 registers, vector
    // loads, one expansion at a time) at every table size.
    std::vector<uint32_t> wpq_choices = {2, 4};
    if (r->want_wpq) wpq_choices = r->want_wpq > 1 ? std::vector<uint32_t>{r->want_wpq} : std::vector<uint32_t>{};
    if (r->want_warps || r->want_regs || r->want_stage || r->want_prefetch || r->want_pipeline == 1)
        wpq_choices.clear();   // those options describe the one-warp kernels
    for (uint32_t q : wpq_choices)
        for (uint32_t b : bit_choices) {
            Tuning c;
            c.wpq = q;
            c.warps = 1;
            c.vh_bits = b;
            c.regs = 2;
            c.stage = 0;
            c.pf = 0;
            c.pipe = 0;
            time_candidate(c);
        }
    // 2. rows loaded ahead, at the best shape (pipelined loop only).
    for (size_t i = 1; i < pf_choices.size() && best.pipe && best.wpq == 1 && a.l0_pipe; ++i) {
        Tuning c = best;
        c.pf = pf_choices[i];
        time_candidate(c);
    }
    // 3. TMA-staged rows at every register budget and warp count, with the
    // best table size found so far.
    for (size_t i = 1; i < stage_choices.size() && r->want_wpq <= 1; ++i) {
        const uint32_t bits = best.vh_bits;
        for (uint32_t reg : reg_choices)
            for (uint32_t w : warp_choices) {
                Tuning c;
                c.warps = w;
                c.vh_bits = bits;
                c.regs = reg;
                c.stage = stage_choices[i];
                c.pf = 0;
                c.pipe = 0;
                time_candidate(c);
            }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    r->tuned[key] = best;
    if (shared && best_ms < 1e29f) tuning_file_store(path, fkey, best);
    return best;
}

int check_kernel_error(artea_gpu_router* r) {
    int h_err = 0;
    CUDA_TRY(cudaMemcpyAsync(&h_err, r->d_error, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    if (h_err != 0) {
        cudaMemsetAsync(r->d_error, 0, sizeof(int), r->stream);
        cudaStreamSynchronize(r->stream);
        static const char* what[] = {"none", "neighbour id out of range", "iteration bound exceeded",
                                     "queue capacity exceeded", "per-query topk/queue outside the router's limits",
                                     "a bulk row copy did not complete within the wait bound"};
        return fail(ARTEA_GPU_EKERNEL, std::string("kernel error: ") + (h_err > 0 && h_err < 6 ? what[h_err] : "?"));
    }
    return ARTEA_GPU_OK;
}

// host_mapped: queries and/or results are page-locked host memory the kernel
// reads and writes in place (their transfers overlap the search); such
// launches read the queries through L2 only and are not captured in graphs,
// whose keys would then follow the caller's buffers.
int run_device(artea_gpu_router* r, const float* d_q, uint32_t nq, const uint32_t* d_topk, const uint32_t* d_queue,
               uint32_t k_stride, uint64_t* d_out, artea_gpu_query_stats* d_stats, bool l0_only, cudaStream_t st,
               bool host_mapped = false) {
    DeviceGuard guard(r->idx->device);
    if (k_stride == 0 && nq) return fail(ARTEA_GPU_EINVAL, "k_stride must be >= topk");
    if (!d_topk && k_stride < r->topk) return fail(ARTEA_GPU_EINVAL, "k_stride must be >= topk");
    if (nq && (!d_q || !d_out)) return fail(ARTEA_GPU_EINVAL, "null query or output buffer");
    if (reinterpret_cast<uintptr_t>(d_q) % 16 != 0 || reinterpret_cast<uintptr_t>(d_out) % 8 != 0)
        return fail(ARTEA_GPU_EINVAL, "queries must be 16-byte and results 8-byte aligned");
    SearchArgs a;
    fill_args(r, &a, d_q, nq, d_topk, d_queue, k_stride, d_out, d_stats, l0_only);
    if (host_mapped) a.coherent = 1;
    bool persistent = r->schedule != ARTEA_GPU_SCHEDULE_PLAIN;
    Tuning t;
    t.warps = 1;
    t.vh_bits = r->want_vh_bits ? hash_bits_of(r->want_vh_bits) : 0;
    t.pf = r->want_prefetch == 16 ? 1u : 0u;
    if (persistent) t = tuned(r, a, st);
    if (r->use_graphs && !host_mapped) return launch_graph(r, a, persistent, t, st);
    return launch_with(r, a, persistent, t, st);
}

// Device address of host memory the GPU reads and writes in place
// (page-locked and mapped, as all page-locked memory is under unified
// addressing), or null for pageable memory.
void* mapped_alias(const void* p) {
    if (!p) return nullptr;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

}  // namespace

namespace artea_gpu {

int index_begin(uint32_t num_vertices, const float* vectors, uint32_t num_vectors, uint32_t dim, int device,
                artea_gpu_index** out) {
    *out = nullptr;
    if (dim == 0 || dim % 16 != 0) return fail(ARTEA_GPU_EINVAL, "dim must be a positive multiple of 16");
    if (num_vectors < num_vertices) return fail(ARTEA_GPU_EINVAL, "fewer vectors than graph vertices");
    if (num_vectors && !vectors) return fail(ARTEA_GPU_EINVAL, "null vectors");
    int ndev = 0;
    if (artea_gpu_device_count(&ndev) != ARTEA_GPU_OK || device < 0 || device >= ndev)
        return fail(ARTEA_GPU_ENODEV, "CUDA device " + std::to_string(device) + " not available");
    DeviceGuard guard(device);
    auto* ix = new artea_gpu_index();
    ix->device = device;
    ix->dim = dim;
    ix->nvecs = num_vectors;
    const size_t nvec = static_cast<size_t>(std::max(num_vectors, 1u)) * dim;
    if (int rc = dev_alloc(&ix->d_vecs, nvec)) {
        artea_gpu_index_destroy(ix);
        return rc;
    }
    if (num_vectors && cudaMemcpy(ix->d_vecs, vectors, sizeof(float) * static_cast<size_t>(num_vectors) * dim,
                                  cudaMemcpyHostToDevice) != cudaSuccess) {
        artea_gpu_index_destroy(ix);
        return fail(ARTEA_GPU_ECUDA, "vector upload failed");
    }
    ix->bytes += sizeof(float) * nvec;
    // x.x of every row, once, for the cosine distance.
    if (int rc = dev_alloc(&ix->d_xsq, std::max(num_vectors, 1u))) {
        artea_gpu_index_destroy(ix);
        return rc;
    }
    ix->bytes += sizeof(float) * std::max(num_vectors, 1u);
    if (num_vectors) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const uint32_t rows_per_block = 8u * 8u;   // 8 warps of 8 rows
        const uint32_t blocks = std::min<uint32_t>((num_vectors + rows_per_block - 1) / rows_per_block,
                                                   static_cast<uint32_t>(std::max(sms, 1)) * 16u);
        row_sqnorm_kernel<<<blocks, 256>>>(ix->d_vecs, num_vectors, dim, ix->d_xsq);
        if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            artea_gpu_index_destroy(ix);
            return fail(ARTEA_GPU_ECUDA, "row norms failed");
        }
    }
    *out = ix;
    return ARTEA_GPU_OK;
}

int index_finish_l0(artea_gpu_index* ix, const uint32_t* vertex_info, const uint64_t* const* group_offsets) {
    // Level-0 row descriptors (start | length << 40), one load per expansion.
    if (ix->n_nbrs >= (1ull << kRowLenShift) || ix->bl >= (1u << 24))
        return fail(ARTEA_GPU_EGRAPH, "graph too large for 40-bit row offsets");
    std::vector<unsigned long long> l0row(ix->n, 0ull);
    for (uint32_t v = 0; v < ix->n; ++v) {
        const uint32_t hl = vertex_info[2 * v];
        if (hl == kInvalidLevel) continue;
        const uint64_t local = vertex_info[2 * v + 1];
        const uint64_t rrow = local * (hl + 1ull) + hl;
        const uint64_t b = group_offsets[hl][rrow], e = group_offsets[hl][rrow + 1];
        l0row[v] = b | ((e - b) << kRowLenShift);
    }
    if (int rc = dev_alloc(&ix->d_l0row, ix->n)) return rc;
    if (cudaMemcpy(ix->d_l0row, l0row.data(), sizeof(unsigned long long) * ix->n, cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return fail(ARTEA_GPU_ECUDA, "row descriptor upload failed");
    ix->bytes += sizeof(uint2) * ix->n + sizeof(uint32_t) * std::max<uint64_t>(ix->n_nbrs, 1) +
                 sizeof(uint64_t) * ix->n_offsets + sizeof(unsigned long long) * ix->n;
    int* d_repeat = nullptr;
    if (int rc = dev_alloc(&d_repeat, 1)) return rc;
    int repeat = 1;
    cudaMemset(d_repeat, 0, sizeof(int));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
    l0_rows_repeat_kernel<<<std::max(sms, 1) * 8, 256>>>(ix->d_l0row, ix->d_nbrs, ix->n, d_repeat);
    const cudaError_t e = cudaMemcpy(&repeat, d_repeat, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(d_repeat);
    if (e != cudaSuccess) return fail(ARTEA_GPU_ECUDA, "row check failed");
    ix->l0_unique = repeat ? 0u : 1u;
    return ARTEA_GPU_OK;
}

}  // namespace artea_gpu

extern "C" {

const char* artea_gpu_version(void) { return "artea-b200 0.1 (sm_100a)"; }

const char* artea_gpu_last_error(void) { return artea_gpu::t_last_error.c_str(); }

int artea_gpu_device_count(int* count) {
    if (!count) return fail(ARTEA_GPU_EINVAL, "null count");
    *count = 0;
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return fail(ARTEA_GPU_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    return ARTEA_GPU_OK;
}

int artea_gpu_index_create(const artea_gpu_graph_desc* g, const float* vectors, uint32_t num_vectors, uint32_t dim,
                           int device, artea_gpu_index** out) {
    if (!g || !out) return fail(ARTEA_GPU_EINVAL, "null argument");
    *out = nullptr;
    if (dim == 0 || dim % 16 != 0) return fail(ARTEA_GPU_EINVAL, "dim must be a positive multiple of 16");
    if (num_vectors < g->num_vertices) return fail(ARTEA_GPU_EINVAL, "fewer vectors than graph vertices");
    if (num_vectors && !vectors) return fail(ARTEA_GPU_EINVAL, "null vectors");
    if (int rc = artea_gpu_graph_validate(g)) return rc;
    artea_gpu_index* ix = nullptr;
    if (int rc = artea_gpu::index_begin(g->num_vertices, vectors, num_vectors, dim, device, &ix)) return rc;
    DeviceGuard guard(device);
    ix->n = g->num_vertices;
    const bool empty = g->num_vertices == 0 || g->top_level == kInvalidLevel;
    ix->top = empty ? kInvalidLevel : g->top_level;
    ix->entry = g->entry_point_vid;
    ix->ul = g->ul_max_nbr_size;
    ix->bl = g->bl_max_nbr_size;
    auto cleanup = [&](int rc) {
        artea_gpu_index_destroy(ix);
        return rc;
    };
    if (!empty) {
        if (int rc = dev_alloc(&ix->d_vinfo, ix->n)) return cleanup(rc);
        if (cudaMemcpy(ix->d_vinfo, g->vertex_info, sizeof(uint2) * ix->n, cudaMemcpyHostToDevice) != cudaSuccess)
            return cleanup(fail(ARTEA_GPU_ECUDA, "vertex table upload failed"));
        ix->n_nbrs = g->num_neighbor_ids;
        const uint64_t nn = std::max<uint64_t>(g->num_neighbor_ids, 1);
        if (int rc = dev_alloc(&ix->d_nbrs, nn)) return cleanup(rc);
        if (g->num_neighbor_ids &&
            cudaMemcpy(ix->d_nbrs, g->neighbor_ids, sizeof(uint32_t) * g->num_neighbor_ids, cudaMemcpyHostToDevice) !=
                cudaSuccess)
            return cleanup(fail(ARTEA_GPU_ECUDA, "neighbour upload failed"));
        uint64_t total = 0;
        for (uint32_t h = 0; h <= ix->top; ++h) total += g->group_sizes[h] * (h + 1ull) + 1;
        ix->n_offsets = total;
        if (int rc = dev_alloc(&ix->d_offsets, total)) return cleanup(rc);
        uint64_t at = 0;
        for (uint32_t h = 0; h <= ix->top; ++h) {
            const uint64_t cnt = g->group_sizes[h] * (h + 1ull) + 1;
            if (cudaMemcpy(ix->d_offsets + at, g->group_offsets[h], sizeof(uint64_t) * cnt, cudaMemcpyHostToDevice) !=
                cudaSuccess)
                return cleanup(fail(ARTEA_GPU_ECUDA, "offset upload failed"));
            ix->group_ptr[h] = ix->d_offsets + at;
            at += cnt;
        }
        if (int rc = artea_gpu::index_finish_l0(ix, g->vertex_info, g->group_offsets)) return cleanup(rc);
    }
    *out = ix;
    return ARTEA_GPU_OK;
}

int artea_gpu_index_destroy(artea_gpu_index* ix) {
    if (!ix) return ARTEA_GPU_OK;
    DeviceGuard guard(ix->device);
    dev_free(ix->d_vecs);
    dev_free(ix->d_xsq);
    dev_free(ix->d_vinfo);
    dev_free(ix->d_nbrs);
    dev_free(ix->d_offsets);
    dev_free(ix->d_l0row);
    delete ix;
    return ARTEA_GPU_OK;
}

int artea_gpu_index_bytes(const artea_gpu_index* ix, uint64_t* bytes) {
    if (!ix || !bytes) return fail(ARTEA_GPU_EINVAL, "null argument");
    *bytes = ix->bytes;
    return ARTEA_GPU_OK;
}

int artea_gpu_router_create(artea_gpu_index* ix, uint32_t topk, uint32_t queue, const artea_gpu_router_opts* opts,
                            artea_gpu_router** out) {
    if (!ix || !out) return fail(ARTEA_GPU_EINVAL, "null argument");
    *out = nullptr;
    if (queue < topk) {
        // hierarchical_graph_router.hpp:104-108
        return fail(ARTEA_GPU_EINVAL, "candidate_queue_size (" + std::to_string(queue) + ") must be >= topk (" +
                                          std::to_string(topk) + ")");
    }
    artea_gpu_router_opts o;
    std::memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    if (o.metric < 0 || o.metric > 3) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    if (o.mode != ARTEA_GPU_MODE_EXACT && o.mode != ARTEA_GPU_MODE_FAST) return fail(ARTEA_GPU_EINVAL, "unknown mode");
    if (o.schedule < 0 || o.schedule > 2) return fail(ARTEA_GPU_EINVAL, "unknown schedule");
    if (o.warps_per_cta > 8) return fail(ARTEA_GPU_EINVAL, "warps_per_cta must be <= 8");
    if (o.register_budget != 0 && o.register_budget != 64 && o.register_budget != 85 && o.register_budget != 96 &&
        o.register_budget != 128)
        return fail(ARTEA_GPU_EINVAL, "register_budget must be 0 (autotuned), 64, 85, 96 or 128");
    if (o.visited_hash_bits != 0 && o.visited_hash_bits != 0xffffffffu &&
        (o.visited_hash_bits < 6 || o.visited_hash_bits > 12))
        return fail(ARTEA_GPU_EINVAL, "visited_hash_bits must be 0 (autotuned), ~0 (no table) or in [6, 12]");
    if (o.stage_rows != 0 && o.stage_rows != 0xffffffffu && o.stage_rows != kStageRows)
        return fail(ARTEA_GPU_EINVAL, "stage_rows must be 0 (autotuned), ~0 (vector loads) or 8");
    if (o.pipeline != 0 && o.pipeline != 1 && o.pipeline != 0xffffffffu)
        return fail(ARTEA_GPU_EINVAL, "pipeline must be 0 (where the graph allows), 1 or ~0 (off)");
    if (o.prefetch_rows != 0 && o.prefetch_rows != 8 && o.prefetch_rows != 16)
        return fail(ARTEA_GPU_EINVAL, "prefetch_rows must be 0 (autotuned), 8 or 16");
    if (o.order_queries != 0 && o.order_queries != 0xffffffffu)
        return fail(ARTEA_GPU_EINVAL, "order_queries must be 0 (largest queue first) or ~0 (index order)");
    if (o.warps_per_query != 0 && o.warps_per_query != 1 && o.warps_per_query != 2 && o.warps_per_query != 4)
        return fail(ARTEA_GPU_EINVAL, "warps_per_query must be 0 (autotuned), 1, 2 or 4");
    if (o.queue_slack != 0 && o.queue_slack != 0xffffffffu && o.queue_slack > 4096)
        return fail(ARTEA_GPU_EINVAL, "queue_slack must be 0 (autotuned), 1..4096 (compact) or ~0 (2L)");
    DeviceGuard guard(ix->device);
    auto* r = new artea_gpu_router();
    r->idx = ix;
    r->topk = topk;
    r->queue = queue;
    r->max_queue = std::max(o.max_queue ? o.max_queue : queue, queue);
    r->cap = std::max<uint32_t>(2u * r->max_queue, 2u);
    r->max_batch = o.max_batch ? o.max_batch : 65536;
    r->metric = o.metric;
    r->mode = o.mode;
    r->schedule = o.schedule;
    r->want_warps = o.warps_per_cta;
    r->want_ctas_per_sm = o.ctas_per_sm;
    r->want_vh_bits = o.visited_hash_bits;
    r->want_regs = o.register_budget;
    r->want_stage = o.stage_rows;
    r->want_pipeline = o.pipeline;
    r->want_prefetch = o.prefetch_rows;
    r->want_order = o.order_queries;
    r->want_wpq = o.warps_per_query;
    r->want_slack = o.queue_slack;
    r->use_graphs = o.use_graphs != 0;
    r->words_per_slot = ((static_cast<uint64_t>(ix->n) + 127) / 128) * 4;   // multiple of 4 words
    r->list_cap = std::max<uint32_t>(std::min<uint32_t>(ix->n, 32768), 64);
    auto cleanup = [&](int rc) {
        artea_gpu_router_destroy(r);
        return rc;
    };
    if (cudaDeviceGetAttribute(&r->num_sms, cudaDevAttrMultiProcessorCount, ix->device) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "cannot query SM count"));
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "cannot create stream"));
    if (int rc = dev_alloc(&r->d_counter, 1)) return cleanup(rc);
    if (int rc = dev_alloc(&r->d_error, 1)) return cleanup(rc);
    if (cudaMemsetAsync(r->d_error, 0, sizeof(int), r->stream) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "memset failed"));
    if (cudaStreamSynchronize(r->stream) != cudaSuccess) return cleanup(fail(ARTEA_GPU_ECUDA, "sync failed"));
    *out = r;
    return ARTEA_GPU_OK;
}

int artea_gpu_router_destroy(artea_gpu_router* r) {
    if (!r) return ARTEA_GPU_OK;
    DeviceGuard guard(r->idx->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    clear_graphs(r);
    dev_free(r->d_vis_bits);
    dev_free(r->d_vis_list);
    dev_free(r->d_counter);
    dev_free(r->d_error);
    dev_free(r->d_order);
    dev_free(r->d_overflow);
    dev_free(r->d_queries);
    dev_free(r->d_out);
    dev_free(r->d_topk);
    dev_free(r->d_queue);
    dev_free(r->d_stats);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return ARTEA_GPU_OK;
}

static int host_query(artea_gpu_router* r, const float* queries, uint32_t nq, const uint32_t* topk_pq,
                      const uint32_t* queue_pq, uint32_t k_stride, uint64_t* out, artea_gpu_query_stats* stats,
                      bool l0_only) {
    if (!r) return fail(ARTEA_GPU_EINVAL, "null router");
    if (nq == 0) return ARTEA_GPU_OK;
    if (!queries || !out) return fail(ARTEA_GPU_EINVAL, "null query or output buffer");
    if (nq > r->max_batch) return fail(ARTEA_GPU_EINVAL, "batch larger than the router's max_batch");
    uint32_t kmax = r->topk;
    if (topk_pq || queue_pq) {
        kmax = 0;
        for (uint32_t i = 0; i < nq; ++i) {
            const uint32_t k = topk_pq ? topk_pq[i] : r->topk;
            const uint32_t L = queue_pq ? queue_pq[i] : r->queue;
            if (L < k) return fail(ARTEA_GPU_EINVAL, "query " + std::to_string(i) + ": queue < topk");
            if (L > r->max_queue) return fail(ARTEA_GPU_EINVAL, "query " + std::to_string(i) + ": queue above max_queue");
            kmax = std::max(kmax, k);
        }
    }
    if (k_stride < kmax) return fail(ARTEA_GPU_EINVAL, "k_stride must be >= every topk");
    DeviceGuard guard(r->idx->device);
    if (int rc = ensure_stage(r, nq, k_stride)) return rc;
    cudaStream_t st = r->stream;
    // Page-locked query and result buffers are read and written by the kernel
    // in place, so their transfers overlap the search; pageable ones are
    // staged through device buffers.
    // (The kernel reads query rows as 16-byte vectors and writes 8-byte words.)
    const float* d_q =
        reinterpret_cast<uintptr_t>(queries) % 16 == 0 ? static_cast<const float*>(mapped_alias(queries)) : nullptr;
    uint64_t* d_o = reinterpret_cast<uintptr_t>(out) % 8 == 0 ? static_cast<uint64_t*>(mapped_alias(out)) : nullptr;
    const bool host_mapped = d_q || d_o;
    if (!d_q) {
        CUDA_TRY(cudaMemcpyAsync(r->d_queries, queries, sizeof(float) * static_cast<size_t>(nq) * r->idx->dim,
                                 cudaMemcpyHostToDevice, st));
        d_q = r->d_queries;
    }
    if (topk_pq) CUDA_TRY(cudaMemcpyAsync(r->d_topk, topk_pq, sizeof(uint32_t) * nq, cudaMemcpyHostToDevice, st));
    if (queue_pq) CUDA_TRY(cudaMemcpyAsync(r->d_queue, queue_pq, sizeof(uint32_t) * nq, cudaMemcpyHostToDevice, st));
    if (int rc = run_device(r, d_q, nq, topk_pq ? r->d_topk : nullptr, queue_pq ? r->d_queue : nullptr, k_stride,
                            d_o ? d_o : r->d_out, stats ? r->d_stats : nullptr, l0_only, st, host_mapped))
        return rc;
    if (!d_o)
        CUDA_TRY(cudaMemcpyAsync(out, r->d_out, sizeof(uint64_t) * static_cast<size_t>(nq) * k_stride,
                                 cudaMemcpyDeviceToHost, st));
    if (stats)
        CUDA_TRY(cudaMemcpyAsync(stats, r->d_stats, sizeof(artea_gpu_query_stats) * nq, cudaMemcpyDeviceToHost, st));
    return check_kernel_error(r);
}

int artea_gpu_batch_query(artea_gpu_router* r, const float* queries, uint32_t nq, const uint32_t* topk_pq,
                          const uint32_t* queue_pq, uint32_t k_stride, uint64_t* out, artea_gpu_query_stats* stats) {
    return host_query(r, queries, nq, topk_pq, queue_pq, k_stride, out, stats, false);
}

int artea_gpu_batch_query_l0_only(artea_gpu_router* r, const float* queries, uint32_t nq, uint32_t k_stride,
                                  uint64_t* out, artea_gpu_query_stats* stats) {
    return host_query(r, queries, nq, nullptr, nullptr, k_stride, out, stats, true);
}

int artea_gpu_batch_query_device(artea_gpu_router* r, const float* d_q, uint32_t nq, const uint32_t* d_topk,
                                 const uint32_t* d_queue, uint32_t k_stride, uint64_t* d_out,
                                 artea_gpu_query_stats* d_stats, void* stream) {
    if (!r) return fail(ARTEA_GPU_EINVAL, "null router");
    if (nq > r->max_batch) return fail(ARTEA_GPU_EINVAL, "batch larger than the router's max_batch");
    // NULL is the CUDA default stream, as in every CUDA API.
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return run_device(r, d_q, nq, d_topk, d_queue, k_stride, d_out, d_stats, false, st);
}

int artea_gpu_router_sync(artea_gpu_router* r) {
    if (!r) return fail(ARTEA_GPU_EINVAL, "null router");
    DeviceGuard guard(r->idx->device);
    CUDA_TRY(cudaDeviceSynchronize());
    return check_kernel_error(r);
}

int artea_gpu_router_set_phase_buffer(artea_gpu_router* r, void* d_phase_cycles) {
    if (!r) return fail(ARTEA_GPU_EINVAL, "null router");
    r->d_phase = static_cast<unsigned long long*>(d_phase_cycles);
    return ARTEA_GPU_OK;
}

// _early_stop_thresholds (hierarchical_graph_router.hpp:388-408): per level
// h in [1, top], the configuration's threshold in double, squared for
// EUCLIDEAN_SQR, must stay a positive finite float that does not round to 0.
int artea_gpu_router_set_early_stop(artea_gpu_router* r, const float* level_thresholds, uint32_t n_levels) {
    if (!r) return fail(ARTEA_GPU_EINVAL, "null router");
    float thr[kMaxGroups] = {};
    const bool on = level_thresholds != nullptr && n_levels != 0;
    const uint32_t top = r->idx->top;
    if (on && top != kInvalidLevel && top != 0) {
        if (n_levels <= top)
            return fail(ARTEA_GPU_EINVAL, "early-stop thresholds cover levels [0, " + std::to_string(n_levels) +
                                              ") but the graph's top level is " + std::to_string(top));
        for (uint32_t h = 1; h <= top; ++h) {
            double t = static_cast<double>(level_thresholds[h]);
            if (r->metric == ARTEA_GPU_EUCLIDEAN_SQR) t *= t;
            if (!std::isfinite(t) || t <= 0.0 || t > static_cast<double>(FLT_MAX) || static_cast<float>(t) == 0.0f)
                return fail(ARTEA_GPU_EINVAL, "Early-stop threshold is not representable in query distance units");
            thr[h] = static_cast<float>(t);
        }
    }
    clear_graphs(r);   // captured launches hold the old arguments
    r->early_stop = on;
    std::memcpy(r->es_thr, thr, sizeof(thr));
    return ARTEA_GPU_OK;
}

int artea_gpu_router_tuning(const artea_gpu_router* r, uint32_t* warps_per_cta, uint32_t* visited_hash_bits,
                            uint32_t* register_budget, uint32_t* stage_rows) {
    if (!r || !warps_per_cta || !visited_hash_bits || !register_budget || !stage_rows)
        return fail(ARTEA_GPU_EINVAL, "null argument");
    *warps_per_cta = r->last.warps;
    *visited_hash_bits = r->last.vh_bits;
    *register_budget = regs_budget(r->last.regs);
    *stage_rows = r->last.stage;
    return ARTEA_GPU_OK;
}

int artea_gpu_router_tuning_ext(const artea_gpu_router* r, uint32_t* pipeline, uint32_t* prefetch_rows,
                                uint32_t* ordered, uint32_t* warps_per_query, uint32_t* queue_slack) {
    if (!r || !pipeline || !prefetch_rows || !ordered || !warps_per_query || !queue_slack)
        return fail(ARTEA_GPU_EINVAL, "null argument");
    *queue_slack = r->last.slack;
    *pipeline = r->last_pipe ? 1u : 0u;
    *prefetch_rows = r->last.pf ? 16u : 8u;
    *ordered = r->last_ordered ? 1u : 0u;
    *warps_per_query = r->last.wpq;
    return ARTEA_GPU_OK;
}

int artea_gpu_router_last_reruns(artea_gpu_router* r, uint32_t* reruns) {
    if (!r || !reruns) return fail(ARTEA_GPU_EINVAL, "null argument");
    *reruns = 0;
    if (!r->d_overflow || !r->last.slack) return ARTEA_GPU_OK;
    DeviceGuard guard(r->idx->device);
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(reruns, r->d_overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return ARTEA_GPU_OK;
}

int artea_gpu_router_launches(const artea_gpu_router* r, uint64_t* launches) {
    if (!r || !launches) return fail(ARTEA_GPU_EINVAL, "null argument");
    *launches = r->launches;
    return ARTEA_GPU_OK;
}

}  // extern "C"

// ===========================================================================
// Batch query that allocates nothing.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside
// a framework's caching allocator or memory-pool callback (where a nested
// allocation would re-enter the allocator), a serving thread that has
// reserved every byte of device memory up front and treats any new
// allocation as a fault, or a plugin whose host process forbids device
// allocation after start-up. artea_gpu_batch_query_noalloc serves them: it
// searches an already uploaded index with the persistent kernel, taking its
// scratch memory (visited bitsets and lists, the work counter, the error
// word) from g_noalloc_scratch, a fixed 64 MiB array that the CUDA loader
// places on every device that loads this library and that stays there until
// the process exits.
//
// Set-up: the first call on a device (with that device current) resolves the
// array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture. Under lazy module loading (the CUDA default
// since 12.2) the array itself is placed when this library's module first
// loads on the device (that first call, or the first launch of any kernel of
// this library), so make that happen at start-up, before the caller reserves
// its device memory. All calls share the array and it keeps the last
// call's contents, so each call zeroes the part it uses before the launch;
// calls that overlap on the GPU (for example on two streams) race on it and
// must be serialised by the caller. The call waits for its kernel so that it
// can report kernel-side errors.
// ===========================================================================
namespace {
constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr size_t kNoAllocHeader = 256;        // work counter + error word, padded
constexpr uint32_t kNoAllocWarps = 4;
constexpr uint32_t kNoAllocMaxQueue = 1024;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

struct NoAllocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;   // device address of g_noalloc_scratch
    int num_sms = 0;
};

std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];

int noalloc_device(int device, NoAllocDevice** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (device < 0 || device >= 64) return fail(ARTEA_GPU_EINVAL, "device index out of range");
    NoAllocDevice& d = g_noalloc_dev[device];
    if (!d.ready) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return fail(ARTEA_GPU_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                             cudaGetErrorString(e));
        }
        int sms = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        d.scratch = static_cast<unsigned char*>(p);
        d.num_sms = sms;
        d.ready = true;
    }
    *out = &d;
    return ARTEA_GPU_OK;
}

}  // namespace

extern "C" int artea_gpu_batch_query_noalloc(const artea_gpu_index* ix, int metric, int mode, uint32_t topk,
                                             uint32_t queue_size, const float* d_queries, uint32_t nq,
                                             uint32_t k_stride, uint64_t* d_out, void* stream) {
    if (!ix) return fail(ARTEA_GPU_EINVAL, "null index");
    if (metric < 0 || metric > 3) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    if (mode != ARTEA_GPU_MODE_EXACT && mode != ARTEA_GPU_MODE_FAST) return fail(ARTEA_GPU_EINVAL, "unknown mode");
    if (queue_size < topk)
        return fail(ARTEA_GPU_EINVAL, "candidate_queue_size (" + std::to_string(queue_size) + ") must be >= topk (" +
                                          std::to_string(topk) + ")");
    if (queue_size > kNoAllocMaxQueue)
        return fail(ARTEA_GPU_EINVAL, "no-alloc query: queue size above the limit of " +
                                          std::to_string(kNoAllocMaxQueue));
    if (k_stride < topk) return fail(ARTEA_GPU_EINVAL, "k_stride must be >= topk");
    if (nq == 0) return ARTEA_GPU_OK;
    if (!d_queries || !d_out) return fail(ARTEA_GPU_EINVAL, "null query or output buffer");
    if (reinterpret_cast<uintptr_t>(d_queries) % 16 != 0) return fail(ARTEA_GPU_EINVAL, "queries must be 16-byte aligned");
    DeviceGuard guard(ix->device);
    NoAllocDevice* dev = nullptr;
    if (int rc = noalloc_device(ix->device, &dev)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Launch shape: 4 warps per CTA, the 85-register kernel, an 8 KB
    // shared-memory visited table when the vid quotient fits in 15 bits.
    const uint32_t cap = std::max<uint32_t>(2u * queue_size, 2u);
    uint32_t vh_bits = 9;
    uint32_t kb = visited_kbits(ix->n, vh_bits);
    if (!kb) {
        vh_bits = 0;
        kb = visited_kbits(ix->n, 0);
    }
    const uint32_t smem = smem_bytes_per_warp(ix->dim, cap, vh_bits) * kNoAllocWarps;
    if (smem > 227u * 1024u) return fail(ARTEA_GPU_EINVAL, "no-alloc query: queue too large for shared memory");
    KernelFn fn = pick_kernel(metric, mode == ARTEA_GPU_MODE_EXACT, true, 0);
    CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(fn),
                                                           static_cast<int>(kNoAllocWarps * 32), smem));
    if (per_sm <= 0) return fail(ARTEA_GPU_EINVAL, "no-alloc query: kernel does not fit on an SM");

    // Scratch layout: [counter, error | pad to 256] [bitsets: slots x words] [lists: slots x list_cap].
    const uint64_t words = ((static_cast<uint64_t>(ix->n) + 127) / 128) * 4;
    const uint32_t list_cap = std::max<uint32_t>(std::min<uint32_t>(ix->n, 4096), 64);
    const uint64_t per_slot = words * 4 + static_cast<uint64_t>(list_cap) * 4;
    const uint64_t max_slots = (kNoAllocScratchBytes - kNoAllocHeader) / per_slot;
    uint64_t ctas = static_cast<uint64_t>(per_sm) * static_cast<uint64_t>(dev->num_sms);
    ctas = std::min<uint64_t>(ctas, max_slots / kNoAllocWarps);
    ctas = std::min<uint64_t>(ctas, (nq + kNoAllocWarps - 1) / kNoAllocWarps);
    if (ctas == 0)
        return fail(ARTEA_GPU_EINVAL, "no-alloc query: the graph needs " + std::to_string(per_slot * kNoAllocWarps) +
                                          " bytes of scratch per CTA; the limit is 64 MiB");
    const uint64_t slots = ctas * kNoAllocWarps;
    unsigned char* base = dev->scratch;
    uint32_t* d_counter = reinterpret_cast<uint32_t*>(base);
    int* d_error = reinterpret_cast<int*>(base + 4);
    uint32_t* bits = reinterpret_cast<uint32_t*>(base + kNoAllocHeader);
    uint32_t* lists = bits + slots * words;
    // The array keeps the previous call's contents: zero the counter, the
    // error word and the bitsets this launch will use.
    CUDA_TRY(cudaMemsetAsync(base, 0, kNoAllocHeader + slots * words * 4, st));

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
    a.k_stride = k_stride;
    a.cap = cap;
    a.vh_bits = vh_bits;
    a.vk_bits = kb;
    a.out = d_out;
    a.vis_bits = bits;
    a.vis_list = lists;
    a.words_per_slot = words;
    a.list_cap = list_cap;
    a.next_query = d_counter;
    a.error = d_error;
    fn<<<static_cast<unsigned>(ctas), kNoAllocWarps * 32, smem, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    int h_err = 0;
    CUDA_TRY(cudaMemcpyAsync(&h_err, d_error, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (h_err != 0) return fail(ARTEA_GPU_EKERNEL, "kernel error " + std::to_string(h_err) + " in no-alloc query");
    return ARTEA_GPU_OK;
}
