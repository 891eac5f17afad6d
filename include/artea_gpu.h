/*
 * artea_gpu.h — C-ABI of the B200 query path for ARTEA compact hierarchical
 * graphs. Plain pointers and sizes only; every function returns an
 * artea_gpu_status and never throws. Thread safety: one index may be queried
 * from several host threads only with distinct artea_gpu_router handles.
 *
 * What each entry point replaces in the reference (paths relative to the
 * reference project root):
 *
 *   artea_gpu_index_create / _from_hgra  — the caller-owned inputs of
 *       HierarchicalGraphRouter: base_vecs (router ctor,
 *       include/artea/cpu/router/hierarchical_graph_router.hpp:93-109) and the
 *       compact::HierarchicalGraph passed to batch_query
 *       (include/artea/cpu/index/compact_structure/hierarchical_graph.hpp:33-201;
 *       HGRA restore: include/artea/cpu/index/persistence/hierarchical_graph_file_manager.hpp:152).
 *       Uploaded once; device resident afterwards.
 *   artea_gpu_router_create — HierarchicalGraphRouter(base_vecs, dist_func, topk,
 *       candidate_queue_size) + initialize() (hierarchical_graph_router.hpp:93-117):
 *       fails with ARTEA_GPU_EINVAL when queue < topk, as the ctor throws.
 *   artea_gpu_batch_query — batch_query<RandomSeeding=false, enable_early_stop=false>
 *       (hierarchical_graph_router.hpp:293-349): host buffers in and out.
 *   artea_gpu_batch_query_device — the same on device-resident buffers and a
 *       caller stream (no host copies).
 *   artea_gpu_batch_query_l0_only — batch_query_l0_only
 *       (hierarchical_graph_router.hpp:353-385).
 *   artea_gpu_hgra_probe / artea_gpu_hgra_read — HierarchicalGraphFileManager::restore
 *       into caller buffers (hierarchical_graph_file_manager.hpp:15-39, 152-300).
 *   artea_gpu_last_error — text of ARTEA_ERROR / exception messages
 *       (include/artea/common/logger.hpp:97-99).
 *
 * Result words: each result is the 8-byte CandidateEntry
 * (include/artea/cpu/router/data_structures/candidate_entry.hpp:57-65): low 32 bits
 * vid | explored<<31, high 32 bits the float distance. Rows hold k_stride words;
 * unused tail slots hold the invalid entry (vid 0x7FFFFFFF, FLT_MAX)
 * (hierarchical_graph_router.hpp:334, candidate_entry.hpp:97-99).
 */
#ifndef ARTEA_GPU_H
#define ARTEA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum artea_gpu_status {
    ARTEA_GPU_OK = 0,
    ARTEA_GPU_EINVAL = 1,    /* bad argument (sizes, queue < topk, metric, mode) */
    ARTEA_GPU_ENOMEM = 2,    /* device or host allocation failed */
    ARTEA_GPU_ECUDA = 3,     /* a CUDA runtime call failed */
    ARTEA_GPU_EGRAPH = 4,    /* graph failed validation (ids out of range, bad rows) */
    ARTEA_GPU_EIO = 5,       /* snapshot file missing, truncated or malformed */
    ARTEA_GPU_EKERNEL = 6,   /* a kernel reported an internal error (bound exceeded) */
    ARTEA_GPU_ETIMEOUT = 7,  /* a bounded wait gave up */
    ARTEA_GPU_ENODEV = 8,    /* no usable CUDA device */
    ARTEA_GPU_EBUSY = 9      /* serving ring full: poll finished requests first */
} artea_gpu_status;

/* DistanceMetricsT values the router is instantiated with
 * (include/artea/cpu/utils/simd_distance.hpp:64-79). Searches on Euclidean
 * data use EUCLIDEAN_SQR, as search_infra_dispatch maps them
 * (include/artea/cpu/framework/type_context/infra_dispatcher.hpp:234-241). */
typedef enum artea_gpu_metric {
    ARTEA_GPU_EUCLIDEAN_SQR = 0,
    ARTEA_GPU_EUCLIDEAN = 1,
    ARTEA_GPU_COSINE = 2,
    ARTEA_GPU_DOT = 3
} artea_gpu_metric;

/* EXACT reproduces the reference's float summation order (16 lane partials
 * + GCC reduction tree) and its queue's tie rules bit for bit. FAST sums in
 * warp order and merges each neighbour batch into the queue in one step. */
typedef enum artea_gpu_mode {
    ARTEA_GPU_MODE_EXACT = 0,
    ARTEA_GPU_MODE_FAST = 1
} artea_gpu_mode;

/* Kernel schedule. PLAIN: one CTA of one warp per query, grid = nq.
 * PERSISTENT: a grid sized to the GPU whose warps take queries from a shared
 * counter (work stealing); warps_per_cta chosen by the autotuner unless set. */
typedef enum artea_gpu_schedule {
    ARTEA_GPU_SCHEDULE_AUTO = 0,
    ARTEA_GPU_SCHEDULE_PLAIN = 1,
    ARTEA_GPU_SCHEDULE_PERSISTENT = 2
} artea_gpu_schedule;

/* compact::HierarchicalGraph in grouped-CSR form, host memory
 * (include/artea/cpu/index/compact_structure/hierarchical_graph.hpp:46-49, 169-200).
 * Group h lists the vertices whose highest level is h; it has
 * group_sizes[h]*(h+1)+1 offsets, rows ordered level h down to 0 per vertex. */
typedef struct artea_gpu_graph_desc {
    uint32_t num_vertices;
    uint32_t top_level;          /* 0xFFFFFFFF (or num_vertices == 0): empty graph */
    uint32_t ul_max_nbr_size;
    uint32_t bl_max_nbr_size;
    uint32_t entry_point_vid;
    const uint32_t* vertex_info; /* num_vertices x {highest_level, local_vid}; unassigned: {~0u, ~0u} */
    const uint64_t* const* group_offsets; /* top_level+1 pointers */
    const uint64_t* group_sizes; /* top_level+1 vertex counts */
    const uint32_t* neighbor_ids;
    uint64_t num_neighbor_ids;
} artea_gpu_graph_desc;

/* Header of an HGRA v1 snapshot plus the sizes needed to read it. */
typedef struct artea_gpu_hgra_info {
    uint32_t num_vertices;
    uint32_t top_level;
    uint32_t ul_max_nbr_size;
    uint32_t bl_max_nbr_size;
    uint32_t entry_point_vid;
    uint32_t num_groups;         /* top_level + 1 */
    uint64_t num_neighbor_ids;
    uint64_t num_offsets;        /* sum over groups of group_sizes[h]*(h+1)+1 */
    uint64_t group_sizes[64];    /* first num_groups used */
} artea_gpu_hgra_info;

/* Per-query work counters (optional output of a batch query). In EXACT mode
 * they equal the reference's counts: distance calls, rows read per level. */
typedef struct artea_gpu_query_stats {
    uint32_t dist_evals;        /* distance evaluations, entry point included */
    uint32_t upper_rows;        /* neighbour rows read on levels >= 1 (greedy hops) */
    uint32_t upper_row_ids;     /* ids in those rows */
    uint32_t l0_rows;           /* level-0 expansions */
    uint32_t l0_row_ids;        /* ids in level-0 rows */
    uint32_t upper_dist_evals;  /* distance evaluations on levels >= 1 */
    uint32_t results;           /* valid result entries */
    uint32_t visited_spills;    /* visited-list overflows (full bitset clear) */
} artea_gpu_query_stats;

typedef struct artea_gpu_index artea_gpu_index;
typedef struct artea_gpu_router artea_gpu_router;

/* Options of a router (artea_gpu_router_create). Zero-initialise, then set. */
typedef struct artea_gpu_router_opts {
    int metric;              /* artea_gpu_metric */
    int mode;                /* artea_gpu_mode */
    int schedule;            /* artea_gpu_schedule */
    uint32_t warps_per_cta;  /* persistent schedule; 0 = autotuned */
    uint32_t ctas_per_sm;    /* persistent schedule; 0 = as many as fit */
    uint32_t max_batch;      /* largest nq one call may pass; 0 = 65536 */
    uint32_t max_queue;      /* largest per-query queue size; 0 = candidate_queue_size */
    uint32_t use_graphs;     /* capture launches in CUDA graphs and replay them */
    uint32_t visited_hash_bits; /* log2 of the size of the per-warp
                                   shared-memory visited table in 16-byte
                                   units (8 ids per unit, two buckets of 4),
                                   in [6, 12]; 0 = autotuned;
                                   0xFFFFFFFF = no table (HBM bitset only) */
    uint32_t register_budget;   /* registers per thread of the persistent kernel:
                                   64 (32 warps per SM), 85 (80 used, 24
                                   warps), 96 (20 warps) or 128 (16 warps;
                                   96 and 128: CTAs of at most 4 warps);
                                   0 = autotuned */
    uint32_t stage_rows;        /* persistent kernel's row reads: 8 = each pass's
                                   candidate rows staged in shared memory by TMA
                                   bulk copies; 0xFFFFFFFF = vector loads from
                                   HBM/L2; 0 = autotuned */
    uint32_t pipeline;          /* level-0 loop: 1 = pipelined across expansions
                                   where every level-0 row holds at most 64
                                   distinct ids (the next row is collected and
                                   its first rows' loads issued before the
                                   current batch is merged); 0xFFFFFFFF = one
                                   expansion at a time; 0 = autotuned on the
                                   persistent schedule, pipelined on the plain
                                   one */
    uint32_t prefetch_rows;     /* neighbour rows whose loads the pipelined loop
                                   issues ahead of their distance phase: 8 = the
                                   first pass (into registers with the
                                   128-register budget, else into L2), 16 = also
                                   the second pass's rows (into L2);
                                   0 = autotuned */
    uint32_t order_queries;     /* persistent schedule with per-query queue
                                   sizes: 0 = queries are started largest queue
                                   first (longest work first, so the short
                                   queries fill the tail), 0xFFFFFFFF = index
                                   order. Results do not depend on it. */
    uint32_t warps_per_query;   /* persistent schedule: 1 = one warp searches a
                                   query; 2 or 4 = a CTA of that many warps
                                   searches one query, its distance batches
                                   split over the warps (for few, long
                                   searches: small batches, large dims);
                                   0 = autotuned */
    uint32_t queue_slack;       /* persistent one-warp kernels' queue layout:
                                   0xFFFFFFFF = 2L entries per search (room for
                                   every tie of lb the reference keeps);
                                   1..4096 = compact, max queue + that many
                                   entries: a search that could lose a tie of
                                   lb is abandoned and rerun at 2L by a second
                                   kernel on the same stream, so results do
                                   not change; 0 = autotuned (2L or +64) */
} artea_gpu_router_opts;

/* Library / device information. */
const char* artea_gpu_version(void);
const char* artea_gpu_last_error(void);
int artea_gpu_device_count(int* count);

/* ---- HGRA v1 snapshots (host only; no GPU needed) ---- */
int artea_gpu_hgra_probe(const char* path, artea_gpu_hgra_info* info);
/* Fills caller buffers sized from the probe: vertex_info (2*num_vertices u32),
 * offsets (num_offsets u64, groups concatenated in level order), neighbor_ids. */
int artea_gpu_hgra_read(const char* path, uint32_t* vertex_info, uint64_t* offsets, uint32_t* neighbor_ids);
/* Writes an HGRA v1 snapshot of a graph description. */
int artea_gpu_hgra_write(const char* path, const artea_gpu_graph_desc* graph);
/* Checks a graph description on the host (ids in range, rows within their
 * level's capacity, every row id present on that level, monotone offsets). */
int artea_gpu_graph_validate(const artea_gpu_graph_desc* graph);

/* ---- Device-resident index ---- */
/* Validates and uploads the graph and the num_vectors x dim FP32 rows (dim a
 * multiple of 16, rows padded with zeros as the reference pads them). */
int artea_gpu_index_create(const artea_gpu_graph_desc* graph, const float* vectors, uint32_t num_vectors,
                           uint32_t dim, int device, artea_gpu_index** out);
/* Same, restoring the graph from an HGRA v1 snapshot straight to the device;
 * replaces HierarchicalGraphFileManager::restore
 * (index/persistence/hierarchical_graph_file_manager.hpp:152-300) followed by
 * an upload. The file streams through pinned buffers into device memory while
 * the host reads only the record headers; the ids are moved into the compact
 * graph's CSR layout and checked on the device. Same layout, same accepted
 * files and same status codes as artea_gpu_hgra_read + artea_gpu_index_create
 * (EIO for what the reader rejects, EGRAPH for what validation rejects). */
int artea_gpu_index_create_from_hgra(const char* path, const float* vectors, uint32_t num_vectors,
                                     uint32_t dim, int device, artea_gpu_index** out);
/* Copies the device graph back into caller buffers sized as for
 * artea_gpu_hgra_read (vertex_info 2*num_vertices u32, offsets num_offsets
 * u64, neighbor_ids num_neighbor_ids u32); with artea_gpu_hgra_write it
 * snapshots a device index. EINVAL for an index without a graph. */
int artea_gpu_index_download(const artea_gpu_index* index, uint32_t* vertex_info, uint64_t* offsets,
                             uint32_t* neighbor_ids);
int artea_gpu_index_destroy(artea_gpu_index* index);
/* Device bytes held by the index (vectors, their x.x row norms, CSR). */
int artea_gpu_index_bytes(const artea_gpu_index* index, uint64_t* bytes);

/* ---- Router ---- */
/* topk / candidate_queue_size are the defaults used when a call passes no
 * per-query arrays. Fails with EINVAL if candidate_queue_size < topk. */
int artea_gpu_router_create(artea_gpu_index* index, uint32_t topk, uint32_t candidate_queue_size,
                            const artea_gpu_router_opts* opts, artea_gpu_router** out);
int artea_gpu_router_destroy(artea_gpu_router* router);

/* batch_query on host buffers: queries (nq x dim FP32, host) in, out_entries
 * (nq x k_stride words, host) out; k_stride >= every topk. topk_per_query /
 * queue_per_query may be NULL (router defaults). stats (nq, host) may be NULL.
 * Includes the host<->device copies; synchronous. */
int artea_gpu_batch_query(artea_gpu_router* router, const float* queries, uint32_t nq,
                          const uint32_t* topk_per_query, const uint32_t* queue_per_query,
                          uint32_t k_stride, uint64_t* out_entries, artea_gpu_query_stats* stats);

/* Same on device buffers, enqueued on `stream` (a cudaStream_t; NULL = the
 * CUDA default stream); returns without waiting, except on the autotuner's
 * first call: a persistent-schedule router that leaves a launch option to the
 * autotuner times candidate launches on the first call for each (dim, queue
 * capacity, batch-size bucket, per-query arrays) it sees that no earlier
 * process recorded (see artea_gpu_router_opts), on `stream`, and waits for
 * them, so make that call before any stream capture. Buffers must be 16-byte
 * aligned. Per-query arrays and stats are device pointers or NULL. */
int artea_gpu_batch_query_device(artea_gpu_router* router, const float* d_queries, uint32_t nq,
                                 const uint32_t* d_topk, const uint32_t* d_queue, uint32_t k_stride,
                                 uint64_t* d_out, artea_gpu_query_stats* d_stats, void* stream);

/* batch_query_l0_only on host buffers. */
int artea_gpu_batch_query_l0_only(artea_gpu_router* router, const float* queries, uint32_t nq,
                                  uint32_t k_stride, uint64_t* out_entries, artea_gpu_query_stats* stats);

/* Waits for the router's stream and reports any kernel-side error. */
int artea_gpu_router_sync(artea_gpu_router* router);

/* Queries of this router's last compact-queue launch (queue_slack) that were
 * handed to the full-capacity rerun; waits for the device. 0 for other
 * layouts. No reference counterpart (measurement only). */
int artea_gpu_router_last_reruns(artea_gpu_router* router, uint32_t* reruns);

/* Number of kernel launches this router has issued (for launch accounting). */
int artea_gpu_router_launches(const artea_gpu_router* router, uint64_t* launches);

/* Early stop of the upper-level greedy walks: batch_query<RandomSeeding=false,
 * enable_early_stop=true> (hierarchical_graph_router.hpp:176-190, :308-319;
 * thresholds :388-408; the stop test detail/beam_loop.hpp:147-150).
 * level_thresholds[h], h in [1, top], is the graph configuration's
 * early_stop_threshold(h, pruning_config) in its own distance units (index 0
 * is not read); for an EUCLIDEAN_SQR router it is squared, as the reference
 * does. A walk on level h stops once its cursor is at distance <= the
 * threshold; level 0 never stops early. The setting applies to every later
 * launch of this router. level_thresholds NULL (or n_levels 0) switches early
 * stop off. Returns EINVAL when n_levels <= top, or, with the reference's
 * std::overflow_error text "Early-stop threshold is not representable in query
 * distance units", when a converted threshold is non-finite, <= 0, above
 * FLT_MAX or rounds to 0. Graphs that are empty or have no level above 0 need
 * no thresholds (any array is accepted). */
int artea_gpu_router_set_early_stop(artea_gpu_router* router, const float* level_thresholds, uint32_t n_levels);

/* Exact brute-force k-NN over the index's vectors: BruteforceRouter::batch_query
 * (router/bruteforce_router.hpp:130-160) and, with a subset, the subset
 * overload (:164-190, ids are original vector ids). out gets nq rows of topk
 * CandidateEntry words: the min(topk, candidates) nearest in ascending
 * distance (the reference's partial_sort leaves the order of equal distances
 * unspecified; here they come in vid order), then CandidateEntry() padding
 * (vid 0xFFFFFFFF, distance 0). Distances are bit-identical to the reference's
 * SIMD functor. The index may have an empty graph (only its vectors are read).
 * topk in [1, 1024]. subset NULL = all vectors; a non-NULL subset with
 * n_subset 0 gives padding only. The host variant checks subset ids against
 * the vector count (EINVAL) and waits for the result. */
int artea_gpu_bruteforce(const artea_gpu_index* index, int metric, const float* queries, uint32_t nq, uint32_t topk,
                         const uint32_t* subset, uint32_t n_subset, uint64_t* out);

/* The same on device buffers (d_subset ids must be < the vector count); runs on
 * stream (NULL = the default stream) and waits for it before returning. */
int artea_gpu_bruteforce_device(const artea_gpu_index* index, int metric, const float* d_queries, uint32_t nq,
                                uint32_t topk, const uint32_t* d_subset, uint32_t n_subset, uint64_t* d_out,
                                void* stream);

/* The compactor's entry point (hierarchical_graph_compactor.hpp:261-327,
 * _compute_entry_point_vid): the centroid of bucket's vectors (double sums,
 * rounded to float), then the bucket vid nearest to it under metric (the
 * build metric: EUCLIDEAN for L2 graphs). bucket NULL = all vectors; an empty
 * bucket gives 0xFFFFFFFF (invalid_vertex_id). Equal distances resolve to the
 * smallest vid (the reference's parallel reduce leaves them open). EINVAL for
 * ids out of range. Waits for the result. */
int artea_gpu_centroid_entry(const artea_gpu_index* index, int metric, const uint32_t* bucket, uint32_t n,
                             uint32_t* out_vid);

/* Profiling hook: when d_phase_cycles (device memory, nq x 8 uint64) is set,
 * every later launch writes per-query SM clock cycles spent in: greedy upper
 * levels, pop/row lookup, row ids + visited, distances, queue merge, tail,
 * total, and the count of expansions whose row lookup was prefetched. NULL
 * turns it off. No reference counterpart (measurement only). */
int artea_gpu_router_set_phase_buffer(artea_gpu_router* router, void* d_phase_cycles);

/* Subsystem probes (measurement only; no reference counterpart). Runs the
 * query path's subsystems one at a time on the memory accesses of a real
 * search, so that each can be timed and profiled alone: a trace kernel
 * (probe_trace_kernel) searches the nq device queries (EXACT or FAST, one
 * topk and queue for all, visited table of 16 << visited_hash_bits bytes, 0 =
 * none) recording every level-0 expansion, its new candidates and their
 * distances; then (a) the same kernel stops after the upper levels (the
 * greedy descent alone), (d) probe_gather_kernel recomputes the recorded
 * distances in the search's batches, (c) probe_visited_kernel reads every
 * recorded expansion's row and passes it through the visited set, (b)
 * probe_queue_kernel replays the recorded pops and pushes on the queue. Each
 * replay checks itself against the trace (mismatches must be 0). The graph's
 * level-0 rows must hold at most 64 distinct ids. Allocates its trace
 * buffers (about nq * (4096 + 24 * queue) * 8 bytes) and waits. */
typedef struct artea_gpu_probe_result {
    float search_ms;          /* the trace kernel: the whole search */
    float greedy_ms;          /* (a) upper levels only */
    float gather_ms;          /* (d) distance gathers */
    float visited_ms;         /* (c) visited set, with the row reads */
    float queue_ms;           /* (b) queue pops and pushes */
    uint32_t capped_queries;  /* queries whose trace hit its capacity */
    uint64_t candidates;      /* level-0 distance evaluations recorded */
    uint64_t expansions;      /* level-0 expansions recorded */
    uint32_t gather_mismatches, visited_mismatches, queue_mismatches;
} artea_gpu_probe_result;

int artea_gpu_subsystem_probe(const artea_gpu_index* index, int metric, int mode, uint32_t topk,
                              uint32_t queue_size, const float* d_queries, uint32_t nq,
                              uint32_t visited_hash_bits, artea_gpu_probe_result* result);

/* Launch parameters of the router's last launch (the autotuner's choice);
 * stage_rows 0 = vector loads, 8 = TMA-staged rows. */
int artea_gpu_router_tuning(const artea_gpu_router* router, uint32_t* warps_per_cta, uint32_t* visited_hash_bits,
                            uint32_t* register_budget, uint32_t* stage_rows);
/* More of the last launch's parameters: pipelined level-0 loop (0/1),
 * neighbour rows loaded ahead (8 or 16), queries started largest queue first
 * (0/1), warps per query (1, 2, 4), queue slack (0: 2L layout). No reference
 * counterpart (measurement only). */
int artea_gpu_router_tuning_ext(const artea_gpu_router* router, uint32_t* pipeline, uint32_t* prefetch_rows,
                                uint32_t* ordered, uint32_t* warps_per_query, uint32_t* queue_slack);

/* ---- Serving loop (continuous batching) ----
 * No counterpart in the reference, whose batch_query is one blocking call; each
 * query gets the reference's _query (hierarchical_graph_router.hpp:195-248).
 * A server keeps the index, a ring of per-query slots (query row, topk, queue,
 * result row) and one persistent kernel on the device. submit() admits a
 * request of n queries when n ring slots are free (else ARTEA_GPU_EBUSY),
 * copies it in and publishes it to the running kernel, which claims queries
 * one per warp; queries of requests submitted while others run overlap on the
 * device. poll() reports a request done once all its queries are; it copies
 * their rows out and frees the slots. Idle warps read the ring counters without
 * atomics and back off. The kernel stays resident (holding the GPU's warp
 * slots) until the server is destroyed, or until a heartbeat that a thread of
 * the server advances in mapped host memory has not moved for heartbeat_ms:
 * then an idle warp closes the ring and the kernel ends, and submit() and
 * poll() of unfinished work return ARTEA_GPU_ETIMEOUT (destroy the server). So
 * no wait of the kernel outlives a host that stopped answering by more than
 * heartbeat_ms. */
typedef struct artea_gpu_server artea_gpu_server;

typedef struct artea_gpu_server_opts {
    int metric;              /* artea_gpu_metric */
    int mode;                /* artea_gpu_mode */
    uint32_t max_topk;       /* largest topk of any query (result row width) */
    uint32_t max_queue;      /* largest queue size of any query */
    uint32_t ring_slots;     /* queries in flight (admission limit) */
    uint32_t warps_per_cta;  /* 0 = 2 */
    uint32_t idle_polls;     /* must be 0: an idle exit followed by a relaunch on
                                the same stream was seen to leave the new kernel
                                unstarted (cause unknown), so it is refused with
                                ARTEA_GPU_EINVAL */
    uint32_t heartbeat_ms;   /* the kernel ends once the host heartbeat has not
                                moved for this long; 0 = 2000 */
} artea_gpu_server_opts;

int artea_gpu_server_create(artea_gpu_index* index, const artea_gpu_server_opts* opts, artea_gpu_server** out);
/* queries: n x dim host FP32; topk/queue: n per-query values or NULL (the maxima).
 * *ticket identifies the request for poll(). */
int artea_gpu_server_submit(artea_gpu_server* server, const float* queries, uint32_t n, const uint32_t* topk,
                            const uint32_t* queue, uint64_t* ticket);
/* *done = 1 and out_entries (n x k_stride words) filled once every query of the
 * request finished; *done = 0 otherwise. */
int artea_gpu_server_poll(artea_gpu_server* server, uint64_t ticket, uint32_t n, uint32_t k_stride,
                          uint64_t* out_entries, int* done);
int artea_gpu_server_stats(const artea_gpu_server* server, uint64_t* published, uint64_t* consumed,
                           uint64_t* kernel_launches);
int artea_gpu_server_destroy(artea_gpu_server* server);
/* Failure injection on the host: stops this server's heartbeat, as a host
 * that no longer answers would (the kernel ends heartbeat_ms later and
 * unfinished work reports ARTEA_GPU_ETIMEOUT). */
int artea_gpu_server_pause_heartbeat(artea_gpu_server* server);

/* batch_query on device buffers for callers that cannot allocate device
 * memory (inside an allocator callback, under a fully reserved memory pool,
 * or in a host process that forbids allocation after start-up). It allocates
 * nothing: its scratch memory is a fixed 64 MiB array that every GPU loading
 * this library holds until the process exits, so graphs whose per-CTA scratch
 * (4 warps x (N/8 + 16 KiB) bytes) exceeds 64 MiB, and queues above 1024, are
 * rejected with ARTEA_GPU_EINVAL. The array exists once this library's module
 * is loaded on the device; under CUDA's lazy module loading (the default since
 * CUDA 12.2) that happens at the first call or the first launch of any of this
 * library's kernels there, and it takes the array's 64 MiB then. So make one
 * call (or one launch) per device at start-up, before device memory is
 * reserved and before any stream capture; that first call also resolves the
 * array's address. Calls share the array, so calls that overlap on the GPU
 * race. The visited-id lists hold 4,096 ids per search (32,768 in the router),
 * so large searches clear their bitsets whole more often: slower, same
 * results. Waits for its kernel before returning. No counterpart in the
 * reference, whose router always allocates its visited tables and queues on
 * the host. */
int artea_gpu_batch_query_noalloc(const artea_gpu_index* index, int metric, int mode, uint32_t topk,
                                  uint32_t queue_size, const float* d_queries, uint32_t nq, uint32_t k_stride,
                                  uint64_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ARTEA_GPU_H */
