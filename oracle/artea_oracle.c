/*
 * ORACLE — test infrastructure only (see artea_oracle.h). A plain-C
 * restatement of the ARTEA reference query path. Every function names the
 * reference file:line it restates. Compile with -ffp-contract=off and without
 * -ffast-math: the float arithmetic below must round exactly as written.
 */
#define _GNU_SOURCE
#include "artea_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define VID_MASK 0x7FFFFFFFu
#define INVALID_LEVEL 0xFFFFFFFFu
#define ORACLE_MAX_LEVELS 64

/* ---------------------------------------------------------------------------
 * Distances: utils/simd_distance.hpp:64-79 (dispatch), 100-115 + 198 (L2^2,
 * UnrollSize 1), 202-238 (dot), 242-275 (cosine). AVX-512 lane j accumulates
 * elements j, j+16, j+32, ... in chunk order with one fused multiply-add per
 * element, starting from +0. The 16 lanes are then folded by GCC's
 * _mm512_reduce_add_ps tree (avx512fintrin.h __MM512_REDUCE_OP): halves
 * (i, i+8), then (i, i+4), then (i, i^2), then lane 0 + lane 1.
 * ------------------------------------------------------------------------- */
static float reduce16(const float a[16]) {
    float t8[8], t4[4];
    for (int i = 0; i < 8; ++i) t8[i] = a[i + 8] + a[i];
    for (int i = 0; i < 4; ++i) t4[i] = t8[i + 4] + t8[i];
    const float u0 = t4[0] + t4[2];
    const float u1 = t4[1] + t4[3];
    return u0 + u1;
}

static float l2sq(const float* q, const float* x, uint32_t dim) {
    float acc[16] = {0};
    for (uint32_t c = 0; c < dim; c += 16) {
        for (int j = 0; j < 16; ++j) {
            const float d = q[c + j] - x[c + j];
            acc[j] = fmaf(d, d, acc[j]);
        }
    }
    return reduce16(acc);
}

static float dotp(const float* q, const float* x, uint32_t dim) {
    float acc[16] = {0};
    for (uint32_t c = 0; c < dim; c += 16)
        for (int j = 0; j < 16; ++j) acc[j] = fmaf(q[c + j], x[c + j], acc[j]);
    return reduce16(acc);
}

static float cosine(const float* q, const float* x, uint32_t dim) {
    float cross[16] = {0}, n1[16] = {0}, n2[16] = {0};
    for (uint32_t c = 0; c < dim; c += 16) {
        for (int j = 0; j < 16; ++j) {
            const float a = q[c + j], b = x[c + j];
            cross[j] = fmaf(a, b, cross[j]);
            n1[j] = fmaf(a, a, n1[j]);
            n2[j] = fmaf(b, b, n2[j]);
        }
    }
    const float dot = reduce16(cross);
    const float sq1 = reduce16(n1);
    const float sq2 = reduce16(n2);
    const float prod = sq1 * sq2;
    const float denom = sqrtf(prod);
    if (denom > 0.0f) {
        const float ratio = dot / denom;
        return 1.0f - ratio;
    }
    return 1.0f;
}

float oracle_distance(int metric, const float* q, const float* x, uint32_t dim) {
    switch (metric) {
        case ORACLE_EUCLIDEAN_SQR: return l2sq(q, x, dim);
        case ORACLE_EUCLIDEAN: return sqrtf(l2sq(q, x, dim));
        case ORACLE_COSINE: return cosine(q, x, dim);
        case ORACLE_DOT: return -dotp(q, x, dim);
        default: return NAN;
    }
}

/* ---------------------------------------------------------------------------
 * CandidateEntry ordering: router/data_structures/candidate_entry.hpp:170-179
 * (distance first, then the 31-bit vid).
 * ------------------------------------------------------------------------- */
typedef struct entry { uint32_t vid; float dist; } entry;

static int entry_less(entry a, entry b) {
    if (a.dist != b.dist) return a.dist < b.dist;
    return (a.vid & VID_MASK) < (b.vid & VID_MASK);
}

/* Binary heap; max_heap=1 keeps the largest entry on top (std::less),
 * max_heap=0 the smallest (std::greater). Keys are unique (vid), so any
 * correct heap pops the same sequence as std::priority_queue. */
typedef struct heap { entry* a; uint32_t n, cap; int max_heap; } heap;

static int heap_before(const heap* h, entry x, entry y) {
    return h->max_heap ? entry_less(y, x) : entry_less(x, y);
}

static void heap_push(heap* h, entry e) {
    if (h->n == h->cap) {
        h->cap = h->cap ? h->cap * 2 : 64;
        h->a = (entry*)realloc(h->a, sizeof(entry) * h->cap);
    }
    uint32_t i = h->n++;
    h->a[i] = e;
    while (i > 0) {
        uint32_t p = (i - 1) / 2;
        if (!heap_before(h, h->a[i], h->a[p])) break;
        entry t = h->a[i]; h->a[i] = h->a[p]; h->a[p] = t;
        i = p;
    }
}

static entry heap_pop(heap* h) {
    entry top = h->a[0];
    h->a[0] = h->a[--h->n];
    uint32_t i = 0;
    for (;;) {
        uint32_t l = 2 * i + 1, r = l + 1, b = i;
        if (l < h->n && heap_before(h, h->a[l], h->a[b])) b = l;
        if (r < h->n && heap_before(h, h->a[r], h->a[b])) b = r;
        if (b == i) break;
        entry t = h->a[i]; h->a[i] = h->a[b]; h->a[b] = t;
        i = b;
    }
    return top;
}

/* ---------------------------------------------------------------------------
 * StdCandidateQueue: router/data_structures/std_candidate_queue.hpp:68-595.
 * U = unexplored min-heap, T = top-L max-heap, lb = worst distance in T.
 * ------------------------------------------------------------------------- */
typedef struct queue { heap U, T; uint32_t cap; float lb; } queue;

static void queue_init(queue* q, uint32_t cap) {
    q->U.n = 0; q->U.max_heap = 0;
    q->T.n = 0; q->T.max_heap = 1;
    q->cap = cap;
    q->lb = FLT_MAX;
}

/* try_push: std_candidate_queue.hpp:358-388 */
static int queue_try_push(queue* q, uint32_t vid, float dist) {
    entry e = {vid & VID_MASK, dist};
    if (q->T.n >= q->cap && dist >= q->lb) return 0;
    heap_push(&q->U, e);
    heap_push(&q->T, e);
    if (q->T.n > q->cap) (void)heap_pop(&q->T);
    q->lb = q->T.n ? q->T.a[0].dist : FLT_MAX;
    return 1;
}

/* should_terminate: std_candidate_queue.hpp:503-513 */
static int queue_should_terminate(const queue* q) {
    if (q->U.n == 0) return 1;
    if (q->T.n < q->cap) return 0;
    return q->U.a[0].dist > q->lb;
}

/* reset_exploration: std_candidate_queue.hpp:421-426 (U rebuilt from T). */
static void queue_reset_exploration(queue* q) {
    q->U.n = 0;
    for (uint32_t i = 0; i < q->T.n; ++i) heap_push(&q->U, q->T.a[i]);
}

/* ---------------------------------------------------------------------------
 * VersionTagTable: containers/version_tag_table.hpp:47-164. uint16 tag per
 * vid; clear() bumps the version and zeroes the table when it wraps.
 * VisitedTablePool::acquire clears (visited_table_pool.hpp:72).
 * ------------------------------------------------------------------------- */
typedef struct visited { uint16_t* tags; uint32_t n; uint16_t version; } visited;

static void visited_clear(visited* v) {
    v->version++;
    if (v->version == 0) {
        memset(v->tags, 0, sizeof(uint16_t) * v->n);
        v->version = 1;
    }
}
static void visited_set(visited* v, uint32_t i) { v->tags[i] = v->version; }
static int visited_test_and_set(visited* v, uint32_t i) {
    const int was = v->tags[i] == v->version;
    v->tags[i] = v->version;
    return was;
}

/* fetch_level_nbrs: index/compact_structure/hierarchical_graph.hpp:99-108 */
static const uint32_t* level_row(const oracle_graph* g, uint32_t vid, uint32_t level, uint32_t* len) {
    const uint32_t hl = g->vinfo[2 * vid], local = g->vinfo[2 * vid + 1];
    const uint64_t row = (uint64_t)local * ((uint64_t)hl + 1) + (hl - level);
    const uint64_t* off = g->offsets[hl];
    *len = (uint32_t)(off[row + 1] - off[row]);
    return g->nbrs + off[row];
}

typedef struct ctx {
    const oracle_graph* g;
    const float* vecs;
    uint32_t dim;
    int metric;
    visited vis;
    queue q;
    oracle_stats st;
    const float* es_thr;   /* per-level early-stop thresholds (query units) or NULL */
} ctx;

static float dist_of(ctx* c, const float* query, uint32_t vid) {
    c->st.dist_evals++;
    return oracle_distance(c->metric, query, c->vecs + (size_t)vid * c->dim, c->dim);
}

/* greedy_search + greedy_loop_body: single_layer_router.hpp:119-133,
 * detail/beam_loop.hpp:129-166 (first strict improvement in row order). */
static void greedy(ctx* c, const float* query, uint32_t level, uint32_t* cur, float* cur_dist) {
    visited_set(&c->vis, *cur);
    uint32_t best = *cur;
    float best_d = *cur_dist;
    for (;;) {
        /* enable_early_stop: detail/beam_loop.hpp:147-150 (inclusive). */
        if (c->es_thr && best_d <= c->es_thr[level]) break;
        uint32_t next = best;
        float next_d = best_d;
        uint32_t len;
        const uint32_t* row = level_row(c->g, best, level, &len);
        c->st.upper_rows++;
        c->st.upper_row_ids += len;
        for (uint32_t i = 0; i < len; ++i) {
            const uint32_t nb = row[i];
            if (visited_test_and_set(&c->vis, nb)) continue;
            const float d = dist_of(c, query, nb);
            c->st.upper_dist_evals++;
            if (d < next_d) { next_d = d; next = nb; }
        }
        if (next == best) break;
        best = next;
        best_d = next_d;
    }
    *cur = best;
    *cur_dist = best_d;
}

/* beam_search + beam_loop_body: single_layer_router.hpp:145-163,
 * detail/beam_loop.hpp:90-119. process_prefetched_neighbors (beam_loop.hpp:46-75)
 * is order-preserving, so the row is walked in CSR order. */
static void beam(ctx* c, const float* query) {
    queue* q = &c->q;
    queue_reset_exploration(q);
    if (q->U.n == 0) return;
    for (uint32_t i = 0; i < q->T.n; ++i) visited_set(&c->vis, q->T.a[i].vid & VID_MASK);
    while (q->U.n != 0) {
        if (queue_should_terminate(q)) break;
        const entry cur = heap_pop(&q->U);
        if ((cur.vid & VID_MASK) == VID_MASK) break;  /* is_invalid() */
        uint32_t len;
        const uint32_t* row = level_row(c->g, cur.vid & VID_MASK, 0, &len);
        c->st.l0_rows++;
        c->st.l0_row_ids += len;
        for (uint32_t i = 0; i < len; ++i) {
            const uint32_t nb = row[i];
            if (visited_test_and_set(&c->vis, nb)) continue;
            const float d = dist_of(c, query, nb);
            (void)queue_try_push(q, nb, d);
        }
    }
}

static int cmp_entry(const void* a, const void* b) {
    const entry x = *(const entry*)a, y = *(const entry*)b;
    return entry_less(x, y) ? -1 : (entry_less(y, x) ? 1 : 0);
}

/* _query: hierarchical_graph_router.hpp:195-248 (RandomSeeding=false,
 * enable_early_stop=false); l0_only follows query_l0_only (:258-286). */
static uint32_t one_query(ctx* c, const float* query, uint32_t topk, uint32_t L, int l0_only, uint64_t* out) {
    const oracle_graph* g = c->g;
    if (g->num_vertices == 0 || g->top_level == INVALID_LEVEL) return 0;
    visited_clear(&c->vis);  /* VisitedTablePool::acquire */
    uint32_t cur = g->entry_point;
    float cur_d = dist_of(c, query, cur);
    if (!l0_only) {
        for (uint32_t h = g->top_level; h >= 1; --h) {
            greedy(c, query, h, &cur, &cur_d);
            visited_clear(&c->vis);
        }
    }
    queue_init(&c->q, L);
    (void)queue_try_push(&c->q, cur, cur_d);
    beam(c, query);
    const uint32_t k = topk < c->q.T.n ? topk : c->q.T.n;
    if (k == 0) return 0;
    /* extract_results: std_candidate_queue.hpp:542-561 — T ascending, first k. */
    qsort(c->q.T.a, c->q.T.n, sizeof(entry), cmp_entry);
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t dbits;
        memcpy(&dbits, &c->q.T.a[i].dist, 4);
        out[i] = ((uint64_t)dbits << 32) | (c->q.T.a[i].vid & VID_MASK);
    }
    return k;
}

typedef struct job {
    const oracle_graph* g;
    const float* vecs;
    uint32_t dim;
    const float* queries;
    uint32_t nq;
    const uint32_t* topk;
    const uint32_t* queue;
    uint32_t k_stride;
    int metric, l0_only;
    uint64_t* out;
    oracle_stats* stats;
    volatile uint32_t next;
    const float* es_thr;
} job;

static uint64_t invalid_word(void) {
    const float m = FLT_MAX;
    uint32_t bits;
    memcpy(&bits, &m, 4);
    return ((uint64_t)bits << 32) | VID_MASK;
}

static void* worker(void* arg) {
    job* j = (job*)arg;
    ctx c;
    memset(&c, 0, sizeof(c));
    c.g = j->g; c.vecs = j->vecs; c.dim = j->dim; c.metric = j->metric; c.es_thr = j->es_thr;
    c.vis.n = j->g->num_vertices;
    c.vis.tags = (uint16_t*)calloc(c.vis.n ? c.vis.n : 1, sizeof(uint16_t));
    c.vis.version = 1;
    for (;;) {
        const uint32_t i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (i >= j->nq) break;
        memset(&c.st, 0, sizeof(c.st));
        uint64_t* row = j->out + (size_t)i * j->k_stride;
        for (uint32_t r = 0; r < j->k_stride; ++r) row[r] = invalid_word();
        const uint32_t n = one_query(&c, j->queries + (size_t)i * j->dim, j->topk[i], j->queue[i], j->l0_only, row);
        c.st.results = n;
        if (j->stats) j->stats[i] = c.st;
    }
    free(c.vis.tags);
    free(c.q.U.a);
    free(c.q.T.a);
    return NULL;
}

static int run_batch(const oracle_graph* g, const float* vecs, uint32_t dim,
                     const float* queries, uint32_t nq,
                     const uint32_t* topk, const uint32_t* queue, uint32_t k_stride,
                     int metric, int l0_only, uint64_t* out, oracle_stats* stats, int threads,
                     const float* es_thr) {
    if (!g || !out || (nq && (!queries || !topk || !queue)) || dim == 0 || dim % 16) return -1;
    for (uint32_t i = 0; i < nq; ++i)
        if (topk[i] > k_stride || queue[i] < topk[i]) return -1;
    job j = {g, vecs, dim, queries, nq, topk, queue, k_stride, metric, l0_only, out, stats, 0, es_thr};
    if (threads < 1) threads = 1;
    if ((uint32_t)threads > nq) threads = nq ? (int)nq : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    for (int t = 1; t < threads; ++t) pthread_create(&th[t], NULL, worker, &j);
    worker(&j);
    for (int t = 1; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return 0;
}

int oracle_batch_query(const oracle_graph* g, const float* vecs, uint32_t dim,
                       const float* queries, uint32_t nq,
                       const uint32_t* topk, const uint32_t* queue, uint32_t k_stride,
                       int metric, int l0_only, uint64_t* out, oracle_stats* stats, int threads) {
    return run_batch(g, vecs, dim, queries, nq, topk, queue, k_stride, metric, l0_only, out, stats, threads, NULL);
}

/* _early_stop_thresholds: hierarchical_graph_router.hpp:388-408. */
int oracle_early_stop_thresholds(const oracle_graph* g, int metric, const float* cfg, uint32_t n_levels,
                                 float* out) {
    const uint32_t top = g->top_level;
    if (g->num_vertices == 0 || top == INVALID_LEVEL || top == 0) return 0;
    if (!cfg || n_levels <= top) return -1;
    out[0] = 0.0f;
    for (uint32_t h = 1; h <= top; ++h) {
        double t = (double)cfg[h];
        if (metric == ORACLE_EUCLIDEAN_SQR) t *= t;
        if (!isfinite(t) || t <= 0.0 || t > (double)FLT_MAX || (float)t == 0.0f) return -2;
        out[h] = (float)t;
    }
    return 0;
}

int oracle_batch_query_early_stop(const oracle_graph* g, const float* vecs, uint32_t dim,
                                  const float* queries, uint32_t nq,
                                  const uint32_t* topk, const uint32_t* queue, uint32_t k_stride,
                                  int metric, const float* cfg_thresholds, uint32_t n_levels,
                                  uint64_t* out, oracle_stats* stats, int threads) {
    float thr[ORACLE_MAX_LEVELS] = {0};
    if (!g || (g->top_level >= ORACLE_MAX_LEVELS && g->top_level != INVALID_LEVEL)) return -1;
    const int rc = oracle_early_stop_thresholds(g, metric, cfg_thresholds, n_levels, thr);
    if (rc != 0) return rc;
    return run_batch(g, vecs, dim, queries, nq, topk, queue, k_stride, metric, 0, out, stats, threads, thr);
}

/* _compute_entry_point_vid (index/compactor/hierarchical_graph_compactor.hpp:
 * 261-327): double per-dimension sums over the bucket, centroid rounded to
 * float, then the bucket vid with the smallest distance to it (ties: first in
 * bucket order). bucket NULL = [0, n). Returns 0xFFFFFFFF for an empty bucket. */
uint32_t oracle_centroid_entry(const float* vecs, uint32_t dim, const uint32_t* bucket, uint32_t n, int metric) {
    if (n == 0) return 0xFFFFFFFFu;
    double* sums = (double*)calloc(dim, sizeof(double));
    float* c = (float*)malloc(sizeof(float) * dim);
    for (uint32_t i = 0; i < n; ++i) {
        const float* v = vecs + (size_t)(bucket ? bucket[i] : i) * dim;
        for (uint32_t d = 0; d < dim; ++d) sums[d] += (double)v[d];
    }
    const double inv = 1.0 / (double)n;
    for (uint32_t d = 0; d < dim; ++d) c[d] = (float)(sums[d] * inv);
    float best = FLT_MAX;
    uint32_t best_vid = 0xFFFFFFFFu;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t vid = bucket ? bucket[i] : i;
        const float dd = oracle_distance(metric, c, vecs + (size_t)vid * dim, dim);
        if (dd < best) { best = dd; best_vid = vid; }
    }
    free(sums);
    free(c);
    return best_vid;
}

/* ---------------------------------------------------------------------------
 * Exact top-k (router/bruteforce_router.hpp:74-160 idea: full scan + partial
 * sort), ties broken by vid.
 * ------------------------------------------------------------------------- */
typedef struct bf_job {
    const float* vecs; uint32_t n, dim; const float* queries; uint32_t nq, k; int metric;
    uint32_t* ids; float* dists; volatile uint32_t next;
} bf_job;

static void* bf_worker(void* arg) {
    bf_job* j = (bf_job*)arg;
    heap h = {NULL, 0, 0, 1};
    for (;;) {
        const uint32_t qi = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (qi >= j->nq) break;
        const float* q = j->queries + (size_t)qi * j->dim;
        h.n = 0;
        for (uint32_t v = 0; v < j->n; ++v) {
            entry e = {v, oracle_distance(j->metric, q, j->vecs + (size_t)v * j->dim, j->dim)};
            if (h.n < j->k) heap_push(&h, e);
            else if (entry_less(e, h.a[0])) { (void)heap_pop(&h); heap_push(&h, e); }
        }
        const uint32_t m = h.n;
        for (uint32_t r = m; r-- > 0;) {
            entry e = heap_pop(&h);
            j->ids[(size_t)qi * j->k + r] = e.vid;
            j->dists[(size_t)qi * j->k + r] = e.dist;
        }
        for (uint32_t r = m; r < j->k; ++r) {
            j->ids[(size_t)qi * j->k + r] = VID_MASK;
            j->dists[(size_t)qi * j->k + r] = FLT_MAX;
        }
    }
    free(h.a);
    return NULL;
}

int oracle_bruteforce(const float* vecs, uint32_t n, uint32_t dim, const float* queries, uint32_t nq,
                      uint32_t k, int metric, uint32_t* out_ids, float* out_dists, int threads) {
    if (dim == 0 || dim % 16 || k == 0) return -1;
    bf_job j = {vecs, n, dim, queries, nq, k, metric, out_ids, out_dists, 0};
    if (threads < 1) threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    for (int t = 1; t < threads; ++t) pthread_create(&th[t], NULL, bf_worker, &j);
    bf_worker(&j);
    for (int t = 1; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
    return 0;
}
