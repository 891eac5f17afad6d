"""GPU parity of the pipelined level-0 loop and the persistent schedule's
query order.

The pipelined loop decides the next expansion as soon as the current batch's
acceptance is known (the smaller of the first unexplored entry and the
smallest accepted candidate), collects that row and issues its loads before
the current batch is merged. It must return the reference's words, distances
and work counters exactly: here against the one-expansion-at-a-time loop, the
oracle and the golden fixtures, for every register budget (the 128-register
kernel holds the next rows in registers, the others prefetch them into L2),
both prefetch widths, and with queries started largest queue first or in
index order."""
import os
import tempfile

import numpy as np
import pytest

from conftest import BUILDER, build_graph, golden_case
from artea_b200 import datasets as ds
from artea_b200.graph import CompactHierarchicalGraph
from artea_b200.router import DeviceIndex, GpuRouter
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

OFF = 0xFFFFFFFF


@pytest.fixture(scope="module")
def sift20k():
    if not os.path.exists(BUILDER):
        pytest.skip("index builder not built")
    w = ds.WORKLOADS["sift100k"].scaled(20000, 512)
    base, queries = ds.generate(w)
    with tempfile.TemporaryDirectory() as tmp:
        g = CompactHierarchicalGraph.from_hgra(build_graph(base, "euclidean", tmp))
    return g, base, queries


@pytest.fixture(scope="module")
def uneven_ref(sift20k):
    g, base, queries = sift20k
    nq = queries.shape[0]
    rng = np.random.default_rng(17)
    topk = rng.choice(np.array([10, 100], np.uint32), nq)
    queue = np.maximum(rng.choice(np.array([64, 128, 256, 512], np.uint32), nq), topk)
    ref, ost = orc.batch_query(g, base, queries, topk, queue, metric=0, k_stride=100, stats=True)
    return topk, queue, ref, ost


@pytest.mark.parametrize("regs,warps", [(96, 4), (96, 2), (128, 4), (128, 2), (128, 1)])
@pytest.mark.parametrize("prefetch", [8, 16])
def test_pipelined_loop_matches_oracle(sift20k, uneven_ref, regs, warps, prefetch):
    g, base, queries = sift20k
    topk, queue, ref, ost = uneven_ref
    idx = DeviceIndex(g, base)
    r = GpuRouter(idx, 0, 100, 512, mode="exact", schedule="persistent", warps_per_cta=warps, visited_hash_bits=9,
                  register_budget=regs, stage_rows=OFF, prefetch_rows=prefetch)
    out, st = r.batch_query(queries, topk=topk, queue=queue, k_stride=100, stats=True)
    np.testing.assert_array_equal(out, ref, err_msg=f"regs={regs} warps={warps} prefetch={prefetch}")
    np.testing.assert_array_equal(st[:, :7], ost[:, :7])
    t = r.tuning()
    assert t["pipeline"] == 1 and t["prefetch_rows"] == prefetch and t["register_budget"] == regs
    assert t["ordered"] == 1, "per-query queue sizes: largest queue first by default"
    r.close()
    idx.close()


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
def test_pipelined_equals_one_expansion_loop(sift20k, schedule):
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    outs = {}
    for pipe in (1, OFF, 0):
        r = GpuRouter(idx, 0, 100, 200, mode="exact", schedule=schedule, pipeline=pipe, stage_rows=OFF)
        outs[pipe] = r.batch_query(queries, stats=True)
        if pipe != 0:
            assert r.tuning()["pipeline"] == (1 if pipe == 1 else 0)
        r.close()
    ref = orc.batch_query(g, base, queries, 100, 200, metric=0)
    for pipe in (1, OFF, 0):   # pipelined, one expansion at a time, autotuned
        np.testing.assert_array_equal(outs[pipe][0], ref, err_msg=f"pipeline={pipe}")
        np.testing.assert_array_equal(outs[pipe][1][:, :7], outs[1][1][:, :7])
    idx.close()


def test_query_order_does_not_change_results(sift20k, uneven_ref):
    g, base, queries = sift20k
    topk, queue, ref, _ = uneven_ref
    idx = DeviceIndex(g, base)
    for order in (0, OFF):
        for graphs in (False, True):
            r = GpuRouter(idx, 0, 100, 512, mode="exact", schedule="persistent", order_queries=order,
                          use_graphs=graphs, warps_per_cta=2, visited_hash_bits=9, register_budget=96,
                          stage_rows=OFF, prefetch_rows=8)
            for _ in range(2):
                out = r.batch_query(queries, topk=topk, queue=queue, k_stride=100)
                np.testing.assert_array_equal(out, ref, err_msg=f"order={order} graphs={graphs}")
            assert r.tuning()["ordered"] == (1 if order == 0 else 0)
            r.close()
    idx.close()


@pytest.mark.parametrize("name", ["sift2k", "deep1k_cos", "gist400"])
@pytest.mark.parametrize("regs", [96, 128])
def test_pipelined_loop_matches_reference_fixtures(name, regs):
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    for L in c.queues:
        for prefetch in (8, 16):
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent", warps_per_cta=2,
                          visited_hash_bits=8, register_budget=regs, stage_rows=OFF, prefetch_rows=prefetch)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L} regs={regs} pf={prefetch}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L])
            assert r.tuning()["pipeline"] == 1
            r.close()
    idx.close()


def test_fast_mode_pipelined_within_tolerance(sift20k):
    # FAST mode takes the same pipelined loop; it must agree with EXACT on
    # >= 99.9% of top-k ids.
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    ex = GpuRouter(idx, 0, 100, 200, mode="exact", register_budget=128, stage_rows=OFF).batch_query(queries)
    fa = GpuRouter(idx, 0, 100, 200, mode="fast", register_budget=128, stage_rows=OFF).batch_query(queries)
    ev = (ex & np.uint64(0x7FFFFFFF)).astype(np.int64)
    fv = (fa & np.uint64(0x7FFFFFFF)).astype(np.int64)
    agree = sum(len(set(a) & set(b)) for a, b in zip(ev, fv)) / ev.size
    assert agree >= 0.999
    idx.close()


# ---------------------------------------------------------------------------
# Warps per query: a CTA of 2 or 4 warps searches one query, its distance
# batches split over the warps; words, distances and counters are the
# reference's.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("wpq", [2, 4])
def test_warps_per_query_matches_oracle(sift20k, uneven_ref, wpq):
    g, base, queries = sift20k
    topk, queue, ref, ost = uneven_ref
    idx = DeviceIndex(g, base)
    for order in (0, OFF):
        r = GpuRouter(idx, 0, 100, 512, mode="exact", schedule="persistent", warps_per_query=wpq,
                      visited_hash_bits=9, order_queries=order)
        out, st = r.batch_query(queries, topk=topk, queue=queue, k_stride=100, stats=True)
        np.testing.assert_array_equal(out, ref, err_msg=f"warps_per_query={wpq} order={order}")
        np.testing.assert_array_equal(st[:, :7], ost[:, :7])
        assert r.tuning()["warps_per_query"] == wpq
        r.close()
    idx.close()


@pytest.mark.parametrize("name", ["sift2k", "deep1k_cos", "gist400", "repeats", "axis80", "early_stop_top2"])
@pytest.mark.parametrize("wpq", [2, 4])
def test_warps_per_query_matches_reference_fixtures(name, wpq):
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    for L in c.queues:
        for graphs in (False, True):
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent", warps_per_query=wpq,
                          visited_hash_bits=8, use_graphs=graphs)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L} wpq={wpq}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L])
            r.close()
    for cfg, words, calls in c.es:   # enable_early_stop=true fixtures
        for L in c.queues:
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent", warps_per_query=wpq,
                          visited_hash_bits=8)
            r.set_early_stop(cfg)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, words[L], err_msg=f"{name} early stop L={L} wpq={wpq}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), calls[L])
            r.close()
    idx.close()


def test_autotuner_considers_warps_per_query(sift20k):
    # A batch of 64 queries leaves most of the GPU idle; whatever the tuner
    # picks, the words are the oracle's and the pick is reported.
    g, base, queries = sift20k
    idx = DeviceIndex(g, base)
    r = GpuRouter(idx, 0, 100, 200, mode="exact", schedule="persistent")
    out = r.batch_query(queries[:64])
    np.testing.assert_array_equal(out, orc.batch_query(g, base, queries[:64], 100, 200, metric=0))
    assert r.tuning()["warps_per_query"] in (1, 2, 4)
    r.close()
    idx.close()


# ---------------------------------------------------------------------------
# Compact queue layout: max queue + slack entries per search instead of 2L; a
# search that could lose a tie of lb is abandoned and rerun at 2L by a second
# kernel. A slack of 1 or 2 on integer-valued data (many equal distances)
# makes reruns frequent; words and counters must stay the reference's.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["sift2k", "repeats", "axis80", "deep1k_cos"])
@pytest.mark.parametrize("slack", [1, 2, 64])
def test_compact_queue_matches_reference_fixtures(name, slack):
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    reruns = 0
    for L in c.queues:
        for regs, pf in ((96, 8), (128, 16), (85, 8)):
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule="persistent", warps_per_cta=2,
                          visited_hash_bits=8, register_budget=regs, stage_rows=OFF, prefetch_rows=pf,
                          queue_slack=slack)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L} slack={slack} regs={regs}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L])
            assert r.tuning()["queue_slack"] == slack
            reruns += r.last_reruns()
            r.close()
    if slack == 1 and name in ("sift2k", "repeats"):
        assert reruns > 0, "a slack of 1 on tied distances should hand some searches to the rerun"
    idx.close()


@pytest.mark.parametrize("slack", [1, 64])
def test_compact_queue_uneven_batch_matches_oracle(sift20k, uneven_ref, slack):
    g, base, queries = sift20k
    topk, queue, ref, ost = uneven_ref
    idx = DeviceIndex(g, base)
    for graphs in (False, True):
        r = GpuRouter(idx, 0, 100, 512, mode="exact", schedule="persistent", warps_per_cta=4, visited_hash_bits=9,
                      register_budget=96, stage_rows=OFF, prefetch_rows=8, queue_slack=slack, use_graphs=graphs)
        for _ in range(2):
            out, st = r.batch_query(queries, topk=topk, queue=queue, k_stride=100, stats=True)
            np.testing.assert_array_equal(out, ref, err_msg=f"slack={slack} graphs={graphs}")
            np.testing.assert_array_equal(st[:, :7], ost[:, :7])
        if slack == 1:
            assert r.last_reruns() > 0
        r.close()
    idx.close()


# ---------------------------------------------------------------------------
# Subsystem probes: each replay of a recorded search must agree with the
# trace (distances bit for bit, new-candidate counts, pop order), and the
# trace must hold the search's level-0 work as the counters report it.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name,L", [("sift2k", 32), ("sift2k", 100), ("deep1k_cos", 64), ("gist400", 50)])
def test_subsystem_probes_replay_the_search(name, L):
    import torch
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    res = idx.subsystem_probe(d_q, c.queries.shape[0], c.topk, L, c.metric, visited_hash_bits=8)
    assert res["gather_mismatches"] == 0 and res["visited_mismatches"] == 0 and res["queue_mismatches"] == 0, res
    assert res["capped_queries"] == 0
    _, st = orc.batch_query(c.graph, c.base, c.queries, c.topk, L, metric=c.metric, stats=True)
    st = st.astype(np.int64)
    assert res["candidates"] == int((st[:, 0] - 1 - st[:, 5]).sum())
    assert res["expansions"] == int(st[:, 3].sum())
    assert min(res[k] for k in ("search_ms", "greedy_ms", "gather_ms", "visited_ms", "queue_ms")) > 0
    idx.close()


def test_subsystem_probe_rejects_rows_with_repeats():
    import torch
    from artea_b200 import _native as nat
    c = golden_case("repeats")
    idx = DeviceIndex(c.graph, c.base)
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    with pytest.raises(nat.ArteaGpuError):
        idx.subsystem_probe(d_q, c.queries.shape[0], c.topk, 32, c.metric)
    idx.close()
