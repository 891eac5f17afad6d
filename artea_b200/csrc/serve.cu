// Serving loop: continuous batching of query requests into one persistent
// kernel.
//
// The index stays on the device. Requests of any size are admitted while the
// ring has free slots (the per-query memory: query row, topk/queue, result
// row); their queries are copied into the ring and published by advancing a
// device counter (`tail`). A persistent kernel, already running on every SM,
// claims published queries one per warp (`head`, compare-and-swap) and runs
// the same search as batch_query on them, so queries of requests that arrive
// while others are on the GPU overlap on the device. Each warp writes its
// result row and then a sequence-tagged completion word into mapped host
// memory, where poll() finds them without any CUDA call. The kernel stays
// resident until the server is destroyed, or until the library's heartbeat
// (a counter in mapped host memory that a host thread of the server advances
// every few milliseconds) has not moved for heartbeat_ms: an idle warp that
// sees that closes the ring and the kernel ends, so no wait of the kernel
// outlives its host by more than that; submit() and poll() then return
// ARTEA_GPU_ETIMEOUT.
//
// There is no serving loop in the reference (its batch_query is one blocking
// call); the search each query gets is the reference's _query
// (router/hierarchical_graph_router.hpp:195-248), bit for bit in EXACT mode.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

using namespace artea_gpu;

namespace {

struct ServeCtl {
    unsigned long long* head;         // (closed << 32) | next sequence to claim (device; claimed by CAS)
    const volatile uint32_t* tail;    // sequences published so far (device, written by host copies)
    const volatile uint32_t* stop;    // set by the host to end the kernel
    volatile uint32_t* done;          // mapped host memory: done[slot] = seq + 1 when finished
    volatile uint32_t* closed;        // mapped host memory: kClosedIdle / kClosedHeartbeat by the closing warp
    const volatile uint32_t* beat;    // mapped host memory: the host's heartbeat counter
    uint32_t ring;                    // ring slots; slot = seq % ring
    uint32_t idle_limit;              // microseconds without work before the kernel exits (~0: never)
    uint32_t beat_limit_ms;           // the kernel ends once the heartbeat has not moved for this long
};

constexpr uint32_t kClosedIdle = 1u;        // an idle window ended the instance
constexpr uint32_t kClosedHeartbeat = 2u;   // the host's heartbeat went stale

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

template <int kMetric, bool kExact>
__global__ void __launch_bounds__(256, 3) serve_kernel(SearchArgs a, ServeCtl c) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = lane_id();
    const uint32_t wslot = blockIdx.x * (blockDim.x >> 5) + warp;
    const WarpSmem sm = carve(smem + static_cast<size_t>(warp) * warp_smem_words(a.g.dim, a.cap, a.vh_bits),
                              a.g.dim, a.cap);
    // Idle warps only read head and tail (no atomics) and back off, so the
    // few warps with work are not slowed by thousands polling one address.
    // A kernel instance ends as a whole: the first warp idle for idle_limit
    // microseconds closes the ring for it (the high word of head) while it is
    // empty; every warp then exits once its current query is done, and the
    // host relaunches (reopening the ring) when new work is pending. Warps
    // never leave one by one, which would leave a running kernel with too few
    // warps for the next burst.
    const volatile unsigned long long* vhead = c.head;
    unsigned long long idle_since = 0;
    uint32_t backoff = 64;
    uint32_t beat_seen = *c.beat;
    unsigned long long beat_since = global_ns();
    unsigned long long beat_checked = beat_since;
    for (;;) {
        uint32_t seq = 0;
        int state = 0;   // 0: nothing claimed, 1: claimed seq, 2: ring closed
        if (lane == 0) {
            for (int tries = 0; tries < 64; ++tries) {
                const unsigned long long cur = *vhead;
                if (cur >> 32) {
                    state = 2;
                    break;
                }
                const uint32_t h = static_cast<uint32_t>(cur);
                const uint32_t t = *c.tail;
                if (static_cast<int32_t>(t - h) <= 0) break;
                if (atomicCAS(c.head, cur, cur + 1ull) == cur) {
                    seq = h;
                    state = 1;
                    break;
                }
            }
        }
        state = __shfl_sync(kFull, state, 0);
        seq = __shfl_sync(kFull, seq, 0);
        if (state == 2 || *c.stop) break;
        if (state == 0) {
            const unsigned long long now = global_ns();
            if (idle_since == 0) idle_since = now;
            if (now - beat_checked > 10000000ull) {   // read host memory at most every 10 ms
                beat_checked = now;
                const uint32_t beat = *c.beat;
                if (beat != beat_seen) {
                    beat_seen = beat;
                    beat_since = now;
                }
            }
            const bool stale = now - beat_since > 1000000ull * c.beat_limit_ms;
            if (stale || (c.idle_limit != 0xFFFFFFFFu && now - idle_since > 1000ull * c.idle_limit)) {
                if (lane == 0) {
                    const unsigned long long cur = *vhead;
                    const uint32_t t = *c.tail;
                    // A stale heartbeat closes the ring whatever it holds: the
                    // host that would collect the results no longer answers.
                    if (!(cur >> 32) && (stale || static_cast<int32_t>(t - static_cast<uint32_t>(cur)) <= 0) &&
                        atomicCAS(c.head, cur, cur | (1ull << 32)) == cur) {
                        // Tell the host why this instance is ending.
                        *c.closed = stale ? kClosedHeartbeat : kClosedIdle;
                        __threadfence_system();
                    }
                }
                __syncwarp();
                continue;   // the next look sees the closed ring, or new work
            }
            __nanosleep(backoff);
            backoff = min(backoff * 2u, 16384u);
            continue;
        }
        idle_since = 0;
        backoff = 64;
        // The ring row was written before `tail` advanced (one copy stream);
        // order this warp's reads after the observation of `tail`.
        __threadfence();
        const uint32_t slot = seq % c.ring;
        search_one<kMetric, kExact>(a, slot, wslot, sm);
        // Every lane wrote part of the result row: each fences its own stores
        // before lane 0 publishes the completion word.
        __threadfence_system();
        __syncwarp();
        if (lane == 0) c.done[slot] = seq + 1u;
        __syncwarp();
    }
}

using ServeFn = void (*)(SearchArgs, ServeCtl);

template <int kMetric>
ServeFn pick_m(bool exact) {
    return exact ? serve_kernel<kMetric, true> : serve_kernel<kMetric, false>;
}

ServeFn pick_serve(int metric, bool exact) {
    switch (metric) {
        case ARTEA_GPU_EUCLIDEAN_SQR: return pick_m<ARTEA_GPU_EUCLIDEAN_SQR>(exact);
        case ARTEA_GPU_EUCLIDEAN: return pick_m<ARTEA_GPU_EUCLIDEAN>(exact);
        case ARTEA_GPU_COSINE: return pick_m<ARTEA_GPU_COSINE>(exact);
        case ARTEA_GPU_DOT: return pick_m<ARTEA_GPU_DOT>(exact);
        default: return nullptr;
    }
}

}  // namespace

struct artea_gpu_server {
    artea_gpu_index* idx = nullptr;
    int metric = 0, mode = 0;
    uint32_t kmax = 0, qmax = 0, ring = 0, warps = 0, vh_bits = 0, vk_bits = 0, idle_limit = 0;
    uint32_t grid = 0, smem = 0, cap = 0;
    ServeFn fn = nullptr;
    cudaStream_t kstream = nullptr, cstream = nullptr;
    cudaEvent_t kdone = nullptr;
    bool launched = false;
    uint32_t* h_closed = nullptr;       // mapped: the running instance closed its ring (kClosed*)
    uint32_t* d_closed_alias = nullptr;
    uint32_t* h_beat = nullptr;         // mapped: heartbeat counter advanced by beat_thread
    uint32_t* d_beat_alias = nullptr;
    uint32_t beat_limit_ms = 0;
    std::thread beat_thread;
    std::mutex beat_mu;
    std::condition_variable beat_cv;
    bool beat_quit = false;
    std::atomic<bool> beat_paused{false};
    // device ring and control
    float* d_q = nullptr;
    uint32_t* d_topk = nullptr;
    uint32_t* d_queue = nullptr;
    uint32_t* d_ctl = nullptr;       // [head, closed, tail, stop]: head/closed one 64-bit word
    uint32_t* d_vis_bits = nullptr;
    uint32_t* d_vis_list = nullptr;
    int* d_error = nullptr;
    uint64_t words = 0;
    uint32_t list_cap = 0;
    // pinned host memory
    float* h_q = nullptr;            // staging rows (ring x dim)
    uint32_t* h_meta = nullptr;      // staging topk | queue (2 x ring)
    uint64_t* h_out = nullptr;       // mapped: ring x kmax result words
    uint32_t* h_done = nullptr;      // mapped: ring completion words
    uint64_t* d_out_alias = nullptr;
    uint32_t* d_done_alias = nullptr;
    // host bookkeeping
    uint64_t next_seq = 0;           // published
    uint64_t consumed_upto = 0;      // every seq below is consumed
    std::vector<uint8_t> consumed;   // per slot, for seq >= consumed_upto
    uint64_t launches = 0;
    mutable std::mutex mu;
};

namespace {

int launch_serving(artea_gpu_server* s) {
    SearchArgs a;
    std::memset(&a, 0, sizeof(a));
    const artea_gpu_index* ix = s->idx;
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
    a.queries = s->d_q;
    a.nq = s->ring;
    a.topk = s->d_topk;
    a.queue = s->d_queue;
    a.k_stride = s->kmax;
    a.cap = s->cap;
    a.vh_bits = s->vh_bits;
    a.vk_bits = s->vk_bits;
    a.out = s->d_out_alias;
    a.vis_bits = s->d_vis_bits;
    a.vis_list = s->d_vis_list;
    a.words_per_slot = s->words;
    a.list_cap = s->list_cap;
    a.error = s->d_error;
    a.coherent = 1;
    ServeCtl c;
    c.head = reinterpret_cast<unsigned long long*>(s->d_ctl);
    c.tail = s->d_ctl + 2;
    c.stop = s->d_ctl + 3;
    c.done = s->d_done_alias;
    c.closed = s->d_closed_alias;
    c.beat = s->d_beat_alias;
    c.ring = s->ring;
    c.idle_limit = s->idle_limit;
    c.beat_limit_ms = s->beat_limit_ms;
    CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(s->fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(s->smem)));
    // Reopen the ring (the previous instance closed it before exiting); same
    // stream, so after that instance and before this one.
    CUDA_TRY(cudaMemsetAsync(s->d_ctl + 1, 0, sizeof(uint32_t), s->kstream));
    s->fn<<<s->grid, s->warps * 32, s->smem, s->kstream>>>(a, c);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(s->kdone, s->kstream));
    s->launched = true;
    s->launches++;
    return ARTEA_GPU_OK;
}

bool all_done(const artea_gpu_server* s, uint64_t seq0, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t seq = seq0 + i;
        const volatile uint32_t* d = s->h_done + (seq % s->ring);
        if (*d != static_cast<uint32_t>(seq + 1)) return false;
    }
    return true;
}

// Relaunch the kernel if published work is pending and the running instance
// has closed its ring. The instance's own closing flag (mapped host memory)
// decides, not an event on its stream: the new instance is queued on the same
// stream and starts once the old one has drained.
int ensure_running(artea_gpu_server* s) {
    if (*static_cast<volatile uint32_t*>(s->h_closed) == kClosedHeartbeat)
        return fail(ARTEA_GPU_ETIMEOUT, "serving kernel ended: the host heartbeat was stale for " +
                                            std::to_string(s->beat_limit_ms) + " ms; destroy the server");
    if (s->next_seq == s->consumed_upto) return ARTEA_GPU_OK;
    if (s->launched) {
        if (*static_cast<volatile uint32_t*>(s->h_closed) == 0u) return ARTEA_GPU_OK;
        const cudaError_t q = cudaEventQuery(s->kdone);
        if (q != cudaSuccess && q != cudaErrorNotReady)
            return fail(ARTEA_GPU_ECUDA, std::string("serving kernel: ") + cudaGetErrorString(q));
        int h_err = 0;
        CUDA_TRY(cudaMemcpy(&h_err, s->d_error, sizeof(int), cudaMemcpyDeviceToHost));
        if (h_err) return fail(ARTEA_GPU_EKERNEL, "serving kernel error " + std::to_string(h_err));
    }
    // Anything published but not finished needs a running kernel.
    bool pending = false;
    for (uint64_t seq = s->consumed_upto; seq < s->next_seq && !pending; ++seq) {
        if (!s->consumed[seq % s->ring] && s->h_done[seq % s->ring] != static_cast<uint32_t>(seq + 1)) pending = true;
    }
    if (!pending) return ARTEA_GPU_OK;
    *static_cast<volatile uint32_t*>(s->h_closed) = 0u;
    return launch_serving(s);
}

}  // namespace

extern "C" int artea_gpu_server_create(artea_gpu_index* ix, const artea_gpu_server_opts* opts, artea_gpu_server** out) {
    if (!ix || !opts || !out) return fail(ARTEA_GPU_EINVAL, "null argument");
    *out = nullptr;
    const artea_gpu_server_opts& o = *opts;
    if (o.metric < 0 || o.metric > 3) return fail(ARTEA_GPU_EINVAL, "unknown metric");
    if (o.mode != ARTEA_GPU_MODE_EXACT && o.mode != ARTEA_GPU_MODE_FAST) return fail(ARTEA_GPU_EINVAL, "unknown mode");
    if (o.max_topk == 0 || o.max_queue < o.max_topk) return fail(ARTEA_GPU_EINVAL, "need 0 < max_topk <= max_queue");
    if (o.ring_slots == 0) return fail(ARTEA_GPU_EINVAL, "ring_slots must be > 0");
    DeviceGuard guard(ix->device);
    auto* s = new artea_gpu_server();
    auto cleanup = [&](int rc) {
        artea_gpu_server_destroy(s);
        return rc;
    };
    s->idx = ix;
    s->metric = o.metric;
    s->mode = o.mode;
    s->kmax = o.max_topk;
    s->qmax = o.max_queue;
    s->ring = o.ring_slots;
    s->warps = o.warps_per_cta ? o.warps_per_cta : 2;
    if (s->warps > 8) return cleanup(fail(ARTEA_GPU_EINVAL, "warps_per_cta must be <= 8"));
    // The kernel does not end on idle (it ends at destroy, or when the
    // heartbeat goes stale): an instance that ended and a new one queued behind
    // it on the same stream was seen to leave the new one waiting although
    // every warp of the old one had exited, and the cause is not known, so an
    // idle window is refused.
    if (o.idle_polls != 0)
        return cleanup(fail(ARTEA_GPU_EINVAL, "idle_polls must be 0: the idle exit and relaunch are disabled"));
    s->idle_limit = 0xFFFFFFFFu;
    s->beat_limit_ms = o.heartbeat_ms ? o.heartbeat_ms : 2000u;
    s->cap = std::max<uint32_t>(2u * s->qmax, 2u);
    s->vh_bits = 8;
    s->vk_bits = visited_kbits(ix->n, s->vh_bits);
    if (!s->vk_bits) {
        s->vh_bits = 0;
        s->vk_bits = visited_kbits(ix->n, 0);
    }
    s->fn = pick_serve(o.metric, o.mode == ARTEA_GPU_MODE_EXACT);
    s->smem = warp_smem_words(ix->dim, s->cap, s->vh_bits) * 4u * s->warps;
    if (s->smem > 227u * 1024u) return cleanup(fail(ARTEA_GPU_EINVAL, "max_queue too large for shared memory"));
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(s->fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(s->smem)) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "cannot set shared memory size"));
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(s->fn),
                                                      static_cast<int>(s->warps * 32), s->smem) != cudaSuccess ||
        per_sm <= 0)
        return cleanup(fail(ARTEA_GPU_EINVAL, "serving kernel does not fit on an SM"));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
    s->grid = static_cast<uint32_t>(per_sm * sms);
    const uint64_t slots = static_cast<uint64_t>(s->grid) * s->warps;
    s->words = ((static_cast<uint64_t>(ix->n) + 127) / 128) * 4;
    s->list_cap = std::max<uint32_t>(std::min<uint32_t>(ix->n, 32768), 64);
    if (int rc = dev_alloc(&s->d_q, static_cast<size_t>(s->ring) * ix->dim)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_topk, s->ring)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_queue, s->ring)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_ctl, 4)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_error, 1)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_vis_bits, slots * s->words)) return cleanup(rc);
    if (int rc = dev_alloc(&s->d_vis_list, slots * s->list_cap)) return cleanup(rc);
    if (cudaMemset(s->d_ctl, 0, 16) != cudaSuccess || cudaMemset(s->d_error, 0, sizeof(int)) != cudaSuccess ||
        cudaMemset(s->d_vis_bits, 0, slots * s->words * 4) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "memset failed"));
    if (cudaHostAlloc(reinterpret_cast<void**>(&s->h_q), sizeof(float) * s->ring * ix->dim, cudaHostAllocDefault) !=
            cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&s->h_meta), sizeof(uint32_t) * 2 * s->ring, cudaHostAllocDefault) !=
            cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&s->h_out), sizeof(uint64_t) * s->ring * s->kmax, cudaHostAllocMapped) !=
            cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&s->h_done), sizeof(uint32_t) * s->ring, cudaHostAllocMapped) !=
            cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&s->h_closed), sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&s->h_beat), sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ENOMEM, "pinned host allocation failed"));
    std::memset(s->h_done, 0, sizeof(uint32_t) * s->ring);
    *s->h_closed = 0u;
    *s->h_beat = 0u;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_out_alias), s->h_out, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_done_alias), s->h_done, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_closed_alias), s->h_closed, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_beat_alias), s->h_beat, 0) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "mapped host memory unavailable"));
    if (cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->kdone, cudaEventDisableTiming) != cudaSuccess)
        return cleanup(fail(ARTEA_GPU_ECUDA, "stream/event creation failed"));
    s->consumed.assign(s->ring, 0);
    // The heartbeat: advanced 8 times per limit while the server exists.
    const auto period = std::chrono::milliseconds(std::max<uint32_t>(1u, s->beat_limit_ms / 8u));
    s->beat_thread = std::thread([s, period] {
        std::unique_lock<std::mutex> lk(s->beat_mu);
        while (!s->beat_quit) {
            if (!s->beat_paused.load()) *static_cast<volatile uint32_t*>(s->h_beat) += 1u;
            s->beat_cv.wait_for(lk, period);
        }
    });
    *out = s;
    return ARTEA_GPU_OK;
}

extern "C" int artea_gpu_server_pause_heartbeat(artea_gpu_server* s) {
    if (!s) return fail(ARTEA_GPU_EINVAL, "null server");
    s->beat_paused.store(true);
    return ARTEA_GPU_OK;
}

extern "C" int artea_gpu_server_submit(artea_gpu_server* s, const float* queries, uint32_t n, const uint32_t* topk,
                                       const uint32_t* queue, uint64_t* ticket) {
    if (!s || !ticket || (n && !queries)) return fail(ARTEA_GPU_EINVAL, "null argument");
    if (n == 0) return fail(ARTEA_GPU_EINVAL, "empty request");
    std::lock_guard<std::mutex> lk(s->mu);
    DeviceGuard guard(s->idx->device);
    if (n > s->ring) return fail(ARTEA_GPU_EINVAL, "request larger than the ring");
    if (*static_cast<volatile uint32_t*>(s->h_closed) == kClosedHeartbeat) return ensure_running(s);
    if (s->next_seq + n - s->consumed_upto > s->ring) return fail(ARTEA_GPU_EBUSY, "ring full: poll first");
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t k = topk ? topk[i] : s->kmax;
        const uint32_t L = queue ? queue[i] : s->qmax;
        if (k == 0 || k > s->kmax || L < k || L > s->qmax)
            return fail(ARTEA_GPU_EINVAL, "query " + std::to_string(i) + ": need 0 < topk <= max_topk, topk <= queue <= max_queue");
    }
    const uint32_t dim = s->idx->dim;
    const uint64_t seq0 = s->next_seq;
    // Stage into pinned memory, then copy each contiguous ring segment.
    uint32_t done_n = 0;
    while (done_n < n) {
        const uint32_t slot = static_cast<uint32_t>((seq0 + done_n) % s->ring);
        const uint32_t seg = std::min(n - done_n, s->ring - slot);
        std::memcpy(s->h_q + static_cast<size_t>(slot) * dim, queries + static_cast<size_t>(done_n) * dim,
                    sizeof(float) * seg * dim);
        for (uint32_t i = 0; i < seg; ++i) {
            s->h_meta[slot + i] = topk ? topk[done_n + i] : s->kmax;
            s->h_meta[s->ring + slot + i] = queue ? queue[done_n + i] : s->qmax;
            s->consumed[slot + i] = 0;
        }
        CUDA_TRY(cudaMemcpyAsync(s->d_q + static_cast<size_t>(slot) * dim, s->h_q + static_cast<size_t>(slot) * dim,
                                 sizeof(float) * seg * dim, cudaMemcpyHostToDevice, s->cstream));
        CUDA_TRY(cudaMemcpyAsync(s->d_topk + slot, s->h_meta + slot, sizeof(uint32_t) * seg, cudaMemcpyHostToDevice,
                                 s->cstream));
        CUDA_TRY(cudaMemcpyAsync(s->d_queue + slot, s->h_meta + s->ring + slot, sizeof(uint32_t) * seg,
                                 cudaMemcpyHostToDevice, s->cstream));
        done_n += seg;
    }
    // Publish: the new tail value is copied from pageable memory (captured at
    // the call), ordered after the row copies on the same stream.
    uint32_t new_tail = static_cast<uint32_t>(seq0 + n);
    CUDA_TRY(cudaMemcpyAsync(s->d_ctl + 2, &new_tail, sizeof(uint32_t), cudaMemcpyHostToDevice, s->cstream));
    s->next_seq = seq0 + n;
    *ticket = seq0;
    return ensure_running(s);
}

extern "C" int artea_gpu_server_poll(artea_gpu_server* s, uint64_t ticket, uint32_t n, uint32_t k_stride,
                                     uint64_t* out_entries, int* done) {
    if (!s || !done || (n && !out_entries)) return fail(ARTEA_GPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    DeviceGuard guard(s->idx->device);
    *done = 0;
    if (ticket < s->consumed_upto || ticket + n > s->next_seq) return fail(ARTEA_GPU_EINVAL, "unknown ticket");
    if (!all_done(s, ticket, n)) return ensure_running(s);
    const uint32_t k = std::min(k_stride, s->kmax);
    constexpr uint64_t kInvalidWord = (static_cast<uint64_t>(0x7f7fffffu) << 32) | 0x7fffffffu;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t slot = static_cast<uint32_t>((ticket + i) % s->ring);
        const volatile uint64_t* src = s->h_out + static_cast<size_t>(slot) * s->kmax;
        uint64_t* dst = out_entries + static_cast<size_t>(i) * k_stride;
        for (uint32_t j = 0; j < k; ++j) dst[j] = src[j];
        for (uint32_t j = k; j < k_stride; ++j) dst[j] = kInvalidWord;
        s->consumed[slot] = 1;
    }
    while (s->consumed_upto < s->next_seq && s->consumed[s->consumed_upto % s->ring]) {
        s->consumed[s->consumed_upto % s->ring] = 0;
        s->consumed_upto++;
    }
    *done = 1;
    // The request's results are delivered; a stale heartbeat is reported by
    // the next call that needs the kernel.
    const int rc = ensure_running(s);
    return rc == ARTEA_GPU_ETIMEOUT ? ARTEA_GPU_OK : rc;
}

extern "C" int artea_gpu_server_stats(const artea_gpu_server* s, uint64_t* published, uint64_t* consumed,
                                      uint64_t* launches) {
    if (!s || !published || !consumed || !launches) return fail(ARTEA_GPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *published = s->next_seq;
    *consumed = s->consumed_upto;
    *launches = s->launches;
    return ARTEA_GPU_OK;
}

extern "C" int artea_gpu_server_destroy(artea_gpu_server* s) {
    if (!s) return ARTEA_GPU_OK;
    DeviceGuard guard(s->idx->device);
    if (s->beat_thread.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s->beat_mu);
            s->beat_quit = true;
        }
        s->beat_cv.notify_all();
        s->beat_thread.join();
    }
    if (s->d_ctl) {
        const uint32_t one = 1;
        cudaMemcpy(s->d_ctl + 3, &one, sizeof(uint32_t), cudaMemcpyHostToDevice);
    }
    if (s->kstream) cudaStreamSynchronize(s->kstream);
    if (s->cstream) cudaStreamSynchronize(s->cstream);
    dev_free(s->d_q);
    dev_free(s->d_topk);
    dev_free(s->d_queue);
    dev_free(s->d_ctl);
    dev_free(s->d_error);
    dev_free(s->d_vis_bits);
    dev_free(s->d_vis_list);
    if (s->h_q) cudaFreeHost(s->h_q);
    if (s->h_meta) cudaFreeHost(s->h_meta);
    if (s->h_out) cudaFreeHost(s->h_out);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_closed) cudaFreeHost(s->h_closed);
    if (s->h_beat) cudaFreeHost(s->h_beat);
    if (s->kdone) cudaEventDestroy(s->kdone);
    if (s->kstream) cudaStreamDestroy(s->kstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    delete s;
    return ARTEA_GPU_OK;
}
