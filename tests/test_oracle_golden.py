"""The oracle (C restatement) against the reference's own outputs and known answers."""
import numpy as np
import pytest

from conftest import EARLY_STOP_CASES, GOLDEN_CASES, assert_same_knn, golden_case
from oracle import oracle as orc


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_words_and_calls(name):
    c = golden_case(name)
    for L in c.queues:
        out, st = orc.batch_query(c.graph, c.base, c.queries, c.topk, L, metric=c.metric, stats=True, threads=4)
        np.testing.assert_array_equal(out, c.words[L], err_msg=f"{name} L={L}")
        np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.calls[L], err_msg=f"{name} L={L} calls")


@pytest.mark.parametrize("name", [n for n in GOLDEN_CASES if n in ("sift2k", "deep1k_cos", "gist400", "repeats")])
def test_oracle_l0_only_matches_reference(name):
    c = golden_case(name)
    for L in c.queues:
        out, st = orc.batch_query(c.graph, c.base, c.queries, c.topk, L, metric=c.metric, l0_only=True,
                                  stats=True, threads=4)
        np.testing.assert_array_equal(out, c.l0_words[L])
        np.testing.assert_array_equal(st[:, 0].astype(np.uint64), c.l0_calls[L])


def test_early_stop_graph_default_query_makes_seven_distance_calls():
    # unit_tests/test_router_early_stop.cpp:121-129: query = vector 3, topk 1,
    # queue 4 -> result vid 3 after exactly 7 distance calls.
    c = golden_case("early_stop_top2")
    out, st = orc.batch_query(c.graph, c.base, c.queries[3:4], 1, 4, metric=1, stats=True)
    assert (int(out[0, 0]) & 0x7FFFFFFF) == 3
    assert st[0, 0] == 7


def test_early_stop_batch_equals_per_query():
    # test_router_early_stop.cpp:155-157: batch row i returns vid i.
    c = golden_case("early_stop_top2")
    out = orc.batch_query(c.graph, c.base, c.queries, 1, 4, metric=1)
    assert [int(w) & 0x7FFFFFFF for w in out[:, 0]] == [0, 1, 2, 3]


def test_axis80_top10_is_exact_sort_with_ties():
    # test_compact_csr_query.cpp:48-74: results equal an exact sort by
    # (distance, vid), tied distances included.
    c = golden_case("axis80")
    for L in c.queues:
        out = orc.batch_query(c.graph, c.base, c.queries, 10, L, metric=0)
        for i, q in enumerate(c.queries):
            d = np.array([orc.distance(0, q, x) for x in c.base], dtype=np.float32)
            order = sorted(range(80), key=lambda v: (d[v], v))[:10]
            got = [int(w) & 0x7FFFFFFF for w in out[i]]
            if L >= 80:
                assert got == order
            gd = (out[i] >> np.uint64(32)).astype(np.uint32).view(np.float32)
            np.testing.assert_array_equal(gd, d[got])


@pytest.mark.parametrize("dim", [16, 48, 96, 112, 128, 304, 384, 960])
def test_euclidean_known_answer(dim):
    # test_euclidean_distance.cpp:84-98: b = (3, 0, ..., 0, 4) -> 5.
    a = np.zeros(dim, np.float32)
    b = np.zeros(dim, np.float32)
    b[0], b[-1] = 3.0, 4.0
    assert orc.distance(1, a, b) == 5.0
    assert orc.distance(0, a, b) == 25.0
    assert orc.distance(0, a, a) == 0.0


def test_cosine_edge_cases():
    # test_cosine_distance.cpp:90-111.
    rng = np.random.default_rng(7)
    a = rng.standard_normal(96).astype(np.float32)
    assert abs(orc.distance(2, a, a)) < 1e-5
    assert abs(orc.distance(2, a, (a * np.float32(3.5)).astype(np.float32))) < 1e-5
    assert abs(orc.distance(2, a, -a) - 2.0) < 1e-5
    z = np.zeros(96, np.float32)
    assert orc.distance(2, z, a) == 1.0
    assert orc.distance(2, z, z) == 1.0


def test_dot_is_negated_inner_product():
    rng = np.random.default_rng(8)
    a = rng.standard_normal(128).astype(np.float32)
    b = rng.standard_normal(128).astype(np.float32)
    assert abs(orc.distance(3, a, b) + float(np.dot(a.astype(np.float64), b))) < 1e-4


@pytest.mark.parametrize("metric", [0, 1, 2, 3])
@pytest.mark.parametrize("dim", [16, 96, 128, 960])
def test_distance_bit_exact_against_reference_kernel(metric, dim):
    if not orc.have_ref():
        pytest.skip("reference router not built here")
    rng = np.random.default_rng(metric * 1000 + dim)
    for _ in range(50):
        a = (rng.standard_normal(dim) * rng.uniform(0.01, 100)).astype(np.float32)
        b = (rng.standard_normal(dim) * rng.uniform(0.01, 100)).astype(np.float32)
        x = np.float32(orc.distance(metric, a, b))
        y = np.float32(orc.ref_distance(metric, a, b))
        assert x.view(np.uint32) == y.view(np.uint32)


def test_scalar_double_reference_within_tolerance():
    # test_euclidean_distance.cpp:67-82: within 2e-6 relative of a double sum.
    rng = np.random.default_rng(3)
    for dim in (16, 96, 128, 960):
        a = rng.standard_normal(dim).astype(np.float32)
        b = rng.standard_normal(dim).astype(np.float32)
        ref = float(np.sum((a.astype(np.float64) - b) ** 2))
        assert abs(orc.distance(0, a, b) - ref) <= 2e-6 * ref


def test_recall_estimator_semantics():
    # recall_estimator.hpp:150-230: duplicates in predictions count once.
    words = np.array([[1, 1, 2], [5, 6, 7]], dtype=np.uint64)
    gt = np.array([[1, 2, 3], [7, 8, 9]], dtype=np.uint32)
    assert orc.recall_at_k(words, gt, 3) == pytest.approx(3 / 6)


@pytest.mark.parametrize("name", EARLY_STOP_CASES)
def test_oracle_early_stop_matches_reference(name):
    # batch_query<false, true> with per-level configuration thresholds.
    c = golden_case(name)
    assert c.es
    for cfg, words, calls in c.es:
        for L in c.queues:
            out, st = orc.batch_query(c.graph, c.base, c.queries, c.topk, L, metric=c.metric, stats=True,
                                      threads=4, early_stop=cfg)
            np.testing.assert_array_equal(out, words[L], err_msg=f"{name} cfg={cfg} L={L}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), calls[L], err_msg=f"{name} L={L} calls")


def test_early_stop_known_answer_five_calls():
    # test_router_early_stop.cpp:121-135: T_1 = 8, T_2 = 16 -> vid 3, distance
    # 0, 5 distance calls (7 without early stop); L2 and squared L2 alike.
    for name, metric in (("early_stop_top2", 1), ("early_stop_sqr", 0)):
        c = golden_case(name)
        out, st = orc.batch_query(c.graph, c.base, c.queries[3:4], 1, 4, metric=metric, stats=True,
                                  early_stop=[0, 8, 16])
        assert (int(out[0, 0]) & 0x7FFFFFFF) == 3
        assert (int(out[0, 0]) >> 32) == 0
        assert st[0, 0] == 5


def test_early_stop_batch_rows_match_single_queries():
    # test_router_early_stop.cpp:160-180: batch row i returns vid i.
    c = golden_case("early_stop_top2")
    out = orc.batch_query(c.graph, c.base, c.queries, 1, 4, metric=1, early_stop=[0, 8, 16])
    assert [int(w) & 0x7FFFFFFF for w in out[:, 0]] == [0, 1, 2, 3]


def test_early_stop_bottom_only_graph_needs_no_thresholds():
    # test_router_early_stop.cpp:183-197.
    c = golden_case("early_stop_top0")
    out = orc.batch_query(c.graph, c.base, c.queries[3:4], 1, 4, metric=1, early_stop=[])
    assert (int(out[0, 0]) & 0x7FFFFFFF) == 3


@pytest.mark.parametrize("metric,cfg,raises", [
    (0, [0, 1e20, 1e20], True),      # overflows FLT_MAX once squared
    (0, [0, 1e-30, 1e-30], True),    # rounds to 0 once squared
    (0, [0, np.inf, 8], True),
    (0, [0, 8, -1], False),          # squared first: 1 is representable
    (1, [0, 8, -1], True),           # L2 keeps the sign: <= 0
    (1, [0, 0, 8], True),
    (1, [0, 1e-30, 8], False),       # L2 is not squared
])
def test_early_stop_unrepresentable_thresholds(metric, cfg, raises):
    # test_router_early_stop.cpp:200-210 and hierarchical_graph_router.hpp:398-404:
    # thresholds that are not positive finite floats in query units (after
    # squaring for L2^2) raise std::overflow_error; the oracle agrees with the
    # reference on which ones.
    c = golden_case("early_stop_sqr" if metric == 0 else "early_stop_top2")

    def outcome(fn):
        try:
            fn()
            return False
        except orc.EarlyStopNotRepresentable:
            return True

    assert outcome(lambda: orc.batch_query(c.graph, c.base, c.queries, 1, 4, metric=metric, early_stop=cfg)) == raises
    if orc.have_ref():
        r = orc.RefRouter(c.hgra_path, c.base)
        assert outcome(lambda: r.batch_query_early_stop(c.queries, 1, 4, cfg, metric=metric)) == raises
        r.close()


def test_early_stop_thresholds_shorter_than_the_hierarchy_are_rejected():
    c = golden_case("early_stop_top2")
    with pytest.raises(ValueError):
        orc.batch_query(c.graph, c.base, c.queries, 1, 4, metric=1, early_stop=[0, 8])


BRUTEFORCE_CASES = [("early_stop_top2", [1, 3, 10]), ("axis80", [10, 100]), ("sift2k", [10, 100]),
                    ("deep1k_cos", [10, 64]), ("gist400", [10, 50])]


@pytest.mark.parametrize("name,topks", BRUTEFORCE_CASES)
def test_oracle_bruteforce_matches_reference_bruteforce_router(name, topks):
    # bruteforce_router.hpp:74-160: exact distances; equal distances may come in
    # any order in the reference (partial_sort), in vid order in the oracle.
    import numpy as _np
    z = _np.load(f"{__import__('conftest').GOLDEN}/{name}.npz")
    c = golden_case(name)
    for k in topks:
        want = z[f"bf_k{k}"]
        ids, d = orc.bruteforce(c.base, c.queries, k, metric=c.metric, threads=4)
        keff = min(k, c.base.shape[0])
        words = (d.view(_np.uint32).astype(_np.uint64) << _np.uint64(32)) | ids.astype(_np.uint64)
        assert_same_knn(words[:, :keff], want[:, :keff], f"{name} k={k}")
        # the reference pads with CandidateEntry(): vid all ones, distance 0
        assert (want[:, keff:] == _np.uint64(0xFFFFFFFF)).all()


@pytest.mark.parametrize("name,metric", [("sift2k", 1), ("deep1k_cos", 2), ("gist400", 1)])
def test_oracle_centroid_entry_matches_the_reference_compactor(name, metric):
    # hierarchical_graph_compactor.hpp:236-248: the compacted graph's entry
    # point is the top bucket's vid nearest its centroid, under the build
    # metric (true L2 for the Euclidean graphs).
    c = golden_case(name)
    top = c.graph.top_occupied_level_id()
    bucket = np.nonzero(c.graph.vertex_info[:, 0] == top)[0].astype(np.uint32)
    assert orc.centroid_entry(c.base, metric, bucket) == c.graph.entry_point_vid
    assert orc.centroid_entry(c.base, metric, np.zeros(0, np.uint32)) == 0xFFFFFFFF


def _reader_layout(path):
    from artea_b200.graph import CompactHierarchicalGraph
    g = CompactHierarchicalGraph.from_hgra(path)
    offs = np.concatenate(g.group_offsets) if g.num_vertices else np.zeros(0, np.uint64)
    return g.vertex_info, offs, g.neighbor_ids


@pytest.mark.parametrize("name", ["early_stop_top0", "early_stop_top2", "axis80", "sift2k", "deep1k_cos", "gist400"])
def test_snapshot_reader_layout_is_the_references_restore(name):
    # hierarchical_graph_file_manager.hpp:152-300: the reference's restore of
    # the same file gives the same vertex table, group offsets and ids. (The
    # device restore is held to the host reader word for word on the GPU.)
    if not orc.have_ref():
        pytest.skip("reference router not built")
    for got, want in zip(_reader_layout(golden_case(name).hgra_path), orc.ref_restore_layout(golden_case(name).hgra_path)):
        np.testing.assert_array_equal(got, want)


def test_snapshot_reader_layout_on_a_multi_level_snapshot_with_unassigned_vertices(tmp_path):
    from conftest import big_snapshot
    if not orc.have_ref():
        pytest.skip("reference router not built")
    path = str(tmp_path / "big.hgra")
    big_snapshot(path, n=200_000, seed=3)
    for got, want in zip(_reader_layout(path), orc.ref_restore_layout(path)):
        np.testing.assert_array_equal(got, want)
