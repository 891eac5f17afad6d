/*
 * ORACLE — test infrastructure only. A scalar CPU restatement of the ARTEA
 * reference query path, used by tests/, __graft_entry__.smoke() and the CPU
 * baseline arm of bench.py as the checker. Nothing in the product links it.
 *
 * Parity is pinned twice: against the known-answer cases of the reference's
 * own unit tests (restated in tests/golden) and against the reference router
 * itself, compiled from the reference headers into oracle/_ref and run on the
 * same graphs and queries (tests/test_oracle_ref.py).
 */
#ifndef ARTEA_ORACLE_H
#define ARTEA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Metrics, numbered as the product's C-ABI numbers them. */
enum {
    ORACLE_EUCLIDEAN_SQR = 0,
    ORACLE_EUCLIDEAN = 1,
    ORACLE_COSINE = 2,
    ORACLE_DOT = 3
};

/* compact::HierarchicalGraph in its grouped-CSR form
 * (index/compact_structure/hierarchical_graph.hpp:46-49, 169-200). */
typedef struct oracle_graph {
    uint32_t num_vertices;
    uint32_t top_level;          /* 0xFFFFFFFF for an empty graph */
    uint32_t entry_point;
    const uint32_t* vinfo;       /* num_vertices x {highest_level, local_vid} */
    const uint64_t* const* offsets; /* top_level+1 groups; group h has n_h*(h+1)+1 entries */
    const uint32_t* nbrs;
} oracle_graph;

/* Per-query work counters. */
typedef struct oracle_stats {
    uint32_t dist_evals;        /* distance calls, entry point included */
    uint32_t upper_rows;        /* neighbour rows read on levels >= 1 */
    uint32_t upper_row_ids;     /* ids in those rows */
    uint32_t l0_rows;           /* level-0 expansions */
    uint32_t l0_row_ids;        /* ids in level-0 rows */
    uint32_t upper_dist_evals;  /* distance calls on levels >= 1 (entry excluded) */
    uint32_t results;           /* valid result entries written */
    uint32_t reserved;
} oracle_stats;

float oracle_distance(int metric, const float* query, const float* row, uint32_t dim);

/* batch_query of hierarchical_graph_router.hpp:322-349 with RandomSeeding=false
 * and enable_early_stop=false. out has nq rows of k_stride 8-byte
 * CandidateEntry words (low 32 bits vid|explored<<31, high 32 bits float dist),
 * pre-filled with the invalid entry. topk/queue are per-query arrays.
 * Returns 0, or -1 on a bad argument. */
int oracle_batch_query(const oracle_graph* g, const float* vecs, uint32_t dim,
                       const float* queries, uint32_t nq,
                       const uint32_t* topk, const uint32_t* queue, uint32_t k_stride,
                       int metric, int l0_only, uint64_t* out, oracle_stats* stats, int threads);

/* _early_stop_thresholds (hierarchical_graph_router.hpp:388-408): out[h] for
 * h in [1, top] from the configuration's per-level thresholds cfg[h] (squared
 * for EUCLIDEAN_SQR). Returns 0, -1 when cfg covers no more than levels
 * [0, top], -2 when a threshold is not representable in query units (the
 * reference's std::overflow_error). Empty or level-0-only graphs need none. */
int oracle_early_stop_thresholds(const oracle_graph* g, int metric, const float* cfg, uint32_t n_levels,
                                 float* out);

/* batch_query<RandomSeeding=false, enable_early_stop=true>
 * (hierarchical_graph_router.hpp:308-319): as oracle_batch_query, with the
 * greedy walk on level h stopping once its cursor distance is <= the level's
 * threshold (detail/beam_loop.hpp:147-150). Returns the codes of
 * oracle_early_stop_thresholds, or -1 on a bad argument. */
int oracle_batch_query_early_stop(const oracle_graph* g, const float* vecs, uint32_t dim,
                                  const float* queries, uint32_t nq,
                                  const uint32_t* topk, const uint32_t* queue, uint32_t k_stride,
                                  int metric, const float* cfg_thresholds, uint32_t n_levels,
                                  uint64_t* out, oracle_stats* stats, int threads);

/* The compactor's centroid entry point (hierarchical_graph_compactor.hpp:261-327):
 * bucket NULL = vectors [0, n); 0xFFFFFFFF for an empty bucket. */
uint32_t oracle_centroid_entry(const float* vecs, uint32_t dim, const uint32_t* bucket, uint32_t n, int metric);

/* Exact top-k by (distance, vid) over all vectors: ground truth. */
int oracle_bruteforce(const float* vecs, uint32_t n, uint32_t dim, const float* queries, uint32_t nq,
                      uint32_t k, int metric, uint32_t* out_ids, float* out_dists, int threads);

#ifdef __cplusplus
}
#endif

#endif
