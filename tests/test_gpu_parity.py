"""GPU parity: the CUDA path (through the C-ABI) against the reference's own
outputs (golden fixtures) and the oracle on seeded inputs. EXACT mode must be
bit-identical (ids, float distances, distance-call counts); FAST mode must
agree on >= 99.9% of top-k ids with distances within 1e-6 relative."""
import os
import tempfile

import numpy as np
import pytest

from conftest import BUILDER, GOLDEN_CASES, build_graph, golden_case
from artea_b200 import datasets as ds
from artea_b200.graph import CompactHierarchicalGraph
from artea_b200.router import DeviceIndex, GpuRouter, HierarchicalGraphRouter, entry_dists, entry_vids
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

FAST_ID_AGREEMENT = 0.999
# FAST distances agree with EXACT to 1e-6 relative. Cosine distance is
# 1 - dot/|q||x|: near 0 any change of summation order is amplified by the
# cancellation, so for cosine the 1e-6 is taken relative to max(|d|, 1), i.e.
# 1e-6 absolute on its [0, 2] range.
FAST_DIST_RTOL = 1e-6


def fast_dist_ok(d_fast, d_exact, metric):
    scale = max(abs(d_exact), 1.0) if metric == 2 else abs(d_exact)
    return abs(d_fast - d_exact) <= FAST_DIST_RTOL * scale + 1e-30

_indexes = {}


def index_for(name):
    if name not in _indexes:
        c = golden_case(name)
        _indexes[name] = DeviceIndex(c.graph, c.base)
    return _indexes[name]


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_exact_matches_reference_bit_for_bit(name, schedule):
    c = golden_case(name)
    idx = index_for(name)
    for L in c.queues:
        r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule=schedule)
        out, st = r.batch_query(c.queries, stats=True)
        np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L} {schedule}")
        np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L], err_msg=f"{name} L={L} calls")
        r.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_exact_counters_match_oracle(name):
    c = golden_case(name)
    idx = index_for(name)
    L = c.queues[-1]
    r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent")
    _, st = r.batch_query(c.queries, stats=True)
    _, ost = orc.batch_query(c.graph, c.base, c.queries, c.topk, L, metric=c.metric, stats=True)
    np.testing.assert_array_equal(st[:, :7], ost[:, :7])


@pytest.mark.parametrize("name", ["sift2k", "deep1k_cos", "gist400", "repeats"])
def test_l0_only_matches_reference(name):
    c = golden_case(name)
    idx = index_for(name)
    for L in c.queues:
        r = GpuRouter(idx, c.metric, c.topk, L, mode="exact")
        out, st = r.batch_query(c.queries, stats=True, l0_only=True)
        np.testing.assert_array_equal(out, c.l0_words[L])
        np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.l0_calls[L])


def test_drop_in_router_surface_matches_reference():
    c = golden_case("sift2k")
    router = HierarchicalGraphRouter(c.base, "euclidean_sqr", topk=10, candidate_queue_size=32)
    router.initialize()
    words = router.batch_query(c.queries, c.graph)
    assert words.shape == (c.queries.shape[0] * 10,)
    np.testing.assert_array_equal(words.reshape(-1, 10), c.words[32])
    one = router.query(c.queries[5], c.graph)
    np.testing.assert_array_equal(one, c.words[32][5])
    router.close()


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
def test_repeated_and_previsited_ids_in_rows(schedule):
    # Level-0 and level-1 rows that repeat ids and name visited ids (the
    # vertex itself, the entry point, ids collected from earlier rows),
    # including rows longer than 64 ids: the reference skips a later
    # occurrence and a visited id and marks ids at collection
    # (unit_tests/test_compact_csr_query.cpp:89-146). The index must take the
    # repeated-id path (whole-row collection and the pipelined loop need rows
    # of distinct ids) and return the reference's words and distance calls.
    c = golden_case("repeats")
    idx = index_for("repeats")
    assert max(len(c.graph.fetch_level_nbrs(v, 0)) for v in range(c.graph.num_vertices)) > 64
    for L in c.queues:
        for stage in ((0xFFFFFFFF, 8) if schedule == "persistent" else (0,)):
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule=schedule, stage_rows=stage)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, c.words[L], err_msg=f"L={L} {schedule} stage={stage}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L])
            assert r.tuning()["pipeline"] == 0, "rows with repeated ids must not take the pipelined loop"
            r.close()


def _fast_agreement(exact, fast):
    ev, fv = entry_vids(exact), entry_vids(fast)
    agree = sum(len(set(a) & set(b)) for a, b in zip(ev, fv))
    return agree / ev.size


@pytest.mark.parametrize("name", ["sift2k", "deep1k_cos", "gist400"])
def test_fast_mode_within_tolerance(name):
    c = golden_case(name)
    idx = index_for(name)
    L = c.queues[-1]
    ex = GpuRouter(idx, c.metric, c.topk, L, mode="exact").batch_query(c.queries)
    fa = GpuRouter(idx, c.metric, c.topk, L, mode="fast").batch_query(c.queries)
    assert _fast_agreement(ex, fa) >= FAST_ID_AGREEMENT - 0.02   # tiny fixtures: a single swap is 1/240
    # distances of ids found by both modes agree to 1e-6 relative
    for a, b in zip(ex, fa):
        da = dict(zip(entry_vids(a).tolist(), entry_dists(a).tolist()))
        for v, d in zip(entry_vids(b).tolist(), entry_dists(b).tolist()):
            if v in da:
                assert fast_dist_ok(d, da[v], c.metric), (v, d, da[v])


@pytest.fixture(scope="module")
def sift20k():
    if not os.path.exists(BUILDER):
        pytest.skip("index builder not built")
    w = ds.WORKLOADS["sift100k"].scaled(20000, 512)
    base, queries = ds.generate(w)
    with tempfile.TemporaryDirectory() as tmp:
        g = CompactHierarchicalGraph.from_hgra(build_graph(base, "euclidean", tmp))
    return g, base, queries


def test_uneven_per_query_topk_and_queue_exact(sift20k):
    g, base, queries = sift20k
    nq = queries.shape[0]
    rng = np.random.default_rng(11)
    topk = rng.choice(np.array([10, 100], np.uint32), nq)
    queue = np.maximum(rng.choice(np.array([64, 128, 256, 512], np.uint32), nq), topk)
    idx = DeviceIndex(g, base)
    r = GpuRouter(idx, 0, 100, 512, mode="exact", schedule="persistent")
    out, st = r.batch_query(queries, topk=topk, queue=queue, k_stride=100, stats=True)
    ref, ost = orc.batch_query(g, base, queries, topk, queue, metric=0, k_stride=100, stats=True)
    np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(st[:, :7], ost[:, :7])


@pytest.mark.parametrize("L", [100, 200, 400, 800])
def test_exact_queue_sweep_against_oracle(sift20k, L):
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    for schedule in ("plain", "persistent"):
        r = GpuRouter(idx, 0, 100, L, mode="exact", schedule=schedule)
        out = r.batch_query(queries[:256])
        ref = orc.batch_query(g, base, queries[:256], 100, L, metric=0)
        np.testing.assert_array_equal(out, ref, err_msg=f"L={L} {schedule}")


def test_fast_mode_agreement_and_recall(sift20k):
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    ex = GpuRouter(idx, 0, 100, 200, mode="exact").batch_query(queries)
    fa = GpuRouter(idx, 0, 100, 200, mode="fast").batch_query(queries)
    assert _fast_agreement(ex, fa) >= FAST_ID_AGREEMENT
    gt, _ = orc.bruteforce(base, queries, 100)
    assert abs(orc.recall_at_k(ex, gt, 100) - orc.recall_at_k(fa, gt, 100)) <= 0.002


def test_batch_equals_single_queries():
    c = golden_case("deep1k_cos")
    idx = index_for("deep1k_cos")
    r = GpuRouter(idx, c.metric, c.topk, 64)
    batch = r.batch_query(c.queries)
    for i in range(0, c.queries.shape[0], 7):
        np.testing.assert_array_equal(r.batch_query(c.queries[i:i + 1])[0], batch[i])


def test_repeated_calls_reuse_visited_state_cleanly():
    c = golden_case("sift2k")
    idx = index_for("sift2k")
    r = GpuRouter(idx, c.metric, c.topk, 100, schedule="persistent")
    first = r.batch_query(c.queries)
    for _ in range(3):
        np.testing.assert_array_equal(r.batch_query(c.queries), first)
    np.testing.assert_array_equal(first, c.words[100])


def test_empty_graph_returns_invalid_rows():
    g = CompactHierarchicalGraph(0, 0, 4, 4, 0xFFFFFFFF, np.zeros((0, 2), np.uint32), [np.zeros(1, np.uint64)],
                                 np.zeros(0, np.uint32))
    base = np.zeros((4, 16), np.float32)
    idx = DeviceIndex(g, base)
    r = GpuRouter(idx, 1, 1, 4)
    out = r.batch_query(np.zeros((3, 16), np.float32))
    assert (entry_vids(out) == 0x7FFFFFFF).all()
    assert (entry_dists(out) == np.finfo(np.float32).max).all()


def test_topk_larger_than_found_keeps_invalid_tail():
    c = golden_case("early_stop_top0")
    idx = index_for("early_stop_top0")
    r = GpuRouter(idx, 1, 4, 8)
    out = r.batch_query(c.queries, k_stride=6)
    ref = orc.batch_query(c.graph, c.base, c.queries, 4, 8, metric=1, k_stride=6)
    np.testing.assert_array_equal(out, ref)
    assert (entry_vids(out[:, 4:]) == 0x7FFFFFFF).all()


@pytest.mark.parametrize("vh_bits,regs", [(6, 64), (6, 85), (10, 85), (10, 96)])
def test_exact_with_visited_hash_spill_and_register_budgets(sift20k, vh_bits, regs):
    # vh_bits=6 is a 64-bucket (512-slot) table, so every query here sends
    # ids of full buckets to the HBM bitset; results must not change.
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    for warps in ((2, 4) if regs == 96 else (2, 8)):   # budget 96: CTAs of at most 4 warps
        r = GpuRouter(idx, 0, 100, 200, mode="exact", schedule="persistent", warps_per_cta=warps,
                      visited_hash_bits=vh_bits, register_budget=regs, stage_rows=0xFFFFFFFF)
        out, st = r.batch_query(queries[:200], stats=True)
        ref = orc.batch_query(g, base, queries[:200], 100, 200, metric=0)
        np.testing.assert_array_equal(out, ref, err_msg=f"vh_bits={vh_bits} regs={regs} warps={warps}")
        if vh_bits == 6:
            assert (st[:, 7] > 0).all(), "expected every query to spill to the bitset"
        t = r.tuning()
        assert {k: t[k] for k in ("warps_per_cta", "visited_hash_bits", "register_budget", "stage_rows")} == \
            {"warps_per_cta": warps, "visited_hash_bits": vh_bits, "register_budget": regs, "stage_rows": 0}


@pytest.mark.parametrize("regs", [64, 85, 96])
def test_tma_staged_rows_are_bit_exact(sift20k, regs):
    # Rows staged in shared memory by cp.async.bulk (one copy per row, one
    # mbarrier per warp) must leave ids, distances and counters unchanged.
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    nq = queries.shape[0]
    rng = np.random.default_rng(5)
    topk = rng.choice(np.array([10, 100], np.uint32), nq)
    queue = np.maximum(rng.choice(np.array([64, 128, 256], np.uint32), nq), topk)
    ref, ost = orc.batch_query(g, base, queries, topk, queue, metric=0, k_stride=100, stats=True)
    # ctas_per_sm=1 leaves fewer warps than queries: every warp runs several
    # queries on the same staging mbarrier.
    for warps, vh, ctas in ((2, 8, 0), (4, 0xFFFFFFFF, 0), (2, 8, 1)):
        r = GpuRouter(idx, 0, 100, 256, mode="exact", schedule="persistent", warps_per_cta=warps,
                      visited_hash_bits=vh, register_budget=regs, stage_rows=8, ctas_per_sm=ctas)
        out, st = r.batch_query(queries, topk=topk, queue=queue, k_stride=100, stats=True)
        np.testing.assert_array_equal(out, ref, err_msg=f"staged warps={warps} vh={vh}")
        np.testing.assert_array_equal(st[:, :7], ost[:, :7])
        assert r.tuning()["stage_rows"] == 8
        r.close()


@pytest.mark.parametrize("name", ["deep1k_cos", "gist400", "axis80"])
def test_tma_staged_rows_match_reference(name):
    c = golden_case(name)
    idx = index_for(name)
    for L in c.queues:
        r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent", stage_rows=8)
        out, st = r.batch_query(c.queries, stats=True)
        np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L} staged")
        np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L])
        r.close()


def test_plain_schedule_spill(sift20k):
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    r = GpuRouter(idx, 0, 100, 400, mode="exact", schedule="plain", visited_hash_bits=6)
    out = r.batch_query(queries[:100])
    np.testing.assert_array_equal(out, orc.batch_query(g, base, queries[:100], 100, 400, metric=0))


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
def test_cuda_graph_replay_matches_direct_launches(schedule):
    import torch
    c = golden_case("sift2k")
    idx = index_for("sift2k")
    nq = c.queries.shape[0]
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    g = GpuRouter(idx, c.metric, c.topk, 100, schedule=schedule, use_graphs=True)
    outs = []
    d_out = torch.zeros((nq, c.topk), dtype=torch.int64, device=d_q.device)
    for _ in range(3):   # capture, then two replays of the same graph
        d_out.zero_()
        g.batch_query_device(d_q, nq, c.topk, d_out)
        torch.cuda.synchronize()
        outs.append(d_out.cpu().numpy().view(np.uint64))
    for o in outs:
        np.testing.assert_array_equal(o, c.words[100])
    # host-buffer path through graphs as well
    np.testing.assert_array_equal(g.batch_query(c.queries), c.words[100])
    np.testing.assert_array_equal(g.batch_query(c.queries), c.words[100])
    g.sync()


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
@pytest.mark.parametrize("graphs", [False, True])
def test_page_locked_host_buffers_are_used_in_place(schedule, graphs):
    # artea_gpu_batch_query reads page-locked queries and writes page-locked
    # result rows in place; pageable ones go through device staging. Every mix
    # returns the reference's words.
    import torch
    from artea_b200 import _native as nat
    c = golden_case("sift2k")
    nq = c.queries.shape[0]
    r = GpuRouter(index_for("sift2k"), c.metric, c.topk, 100, mode="exact", schedule=schedule, use_graphs=graphs)
    qp = torch.from_numpy(np.ascontiguousarray(c.queries)).pin_memory().numpy()
    for _ in range(2):
        np.testing.assert_array_equal(r.batch_query(qp), c.words[100])          # both in place
        np.testing.assert_array_equal(r.batch_query(c.queries), c.words[100])   # staged queries
        out = np.full((nq, c.topk + 3), 7, np.uint64)                            # staged results, wider rows
        nat.check(nat.lib().artea_gpu_batch_query(r.handle, nat.ptr(qp), nq, None, None, c.topk + 3, nat.ptr(out),
                                                  None))
        np.testing.assert_array_equal(out[:, :c.topk], c.words[100])
        assert (out[:, c.topk:] == np.uint64((0x7F7FFFFF << 32) | 0x7FFFFFFF)).all()
    r.close()
