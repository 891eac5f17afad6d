"""Early stop of the upper-level greedy walks on the GPU
(batch_query<RandomSeeding=false, enable_early_stop=true>) against the
reference's outputs: words and distance calls bit for bit."""
import numpy as np
import pytest

from conftest import EARLY_STOP_CASES, golden_case
from artea_b200._native import ArteaGpuError
from artea_b200.router import DeviceIndex, GpuRouter, HierarchicalGraphRouter
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

_indexes = {}


def index_for(name):
    if name not in _indexes:
        c = golden_case(name)
        _indexes[name] = DeviceIndex(c.graph, c.base)
    return _indexes[name]


@pytest.mark.parametrize("schedule", ["plain", "persistent"])
@pytest.mark.parametrize("name", EARLY_STOP_CASES)
def test_early_stop_matches_reference(name, schedule):
    c = golden_case(name)
    idx = index_for(name)
    for cfg, words, calls in c.es:
        for L in c.queues:
            r = GpuRouter(idx, c.metric, c.topk, L, mode="exact", schedule=schedule)
            r.set_early_stop(cfg)
            out, st = r.batch_query(c.queries, stats=True)
            np.testing.assert_array_equal(out, words[L], err_msg=f"{name} cfg={cfg} L={L}")
            np.testing.assert_array_equal(st[:, 0].astype(np.uint64), calls[L])
            # switched off again: the enable_early_stop=false results
            r.set_early_stop(None)
            np.testing.assert_array_equal(r.batch_query(c.queries), c.words[L])
            r.close()


def test_early_stop_known_answer_five_calls():
    # test_router_early_stop.cpp:121-135: T_1 = 8, T_2 = 16 -> vid 3 at
    # distance 0 after 5 distance calls.
    for name, metric in (("early_stop_top2", 1), ("early_stop_sqr", 0)):
        c = golden_case(name)
        r = GpuRouter(index_for(name), metric, 1, 4, mode="exact")
        r.set_early_stop([0, 8, 16])
        out, st = r.batch_query(c.queries[3:4], stats=True)
        assert (int(out[0, 0]) & 0x7FFFFFFF) == 3 and (int(out[0, 0]) >> 32) == 0
        assert st[0, 0] == 5
        r.close()


@pytest.mark.parametrize("metric,cfg,raises", [
    (0, [0, 1e20, 1e20], True),
    (0, [0, 1e-30, 1e-30], True),
    (0, [0, np.inf, 8], True),
    (0, [0, 8, -1], False),
    (1, [0, 8, -1], True),
    (1, [0, 0, 8], True),
    (1, [0, 1e-30, 8], False),
])
def test_unrepresentable_thresholds_raise_like_the_reference(metric, cfg, raises):
    c = golden_case("early_stop_sqr" if metric == 0 else "early_stop_top2")
    r = GpuRouter(index_for(c.name), metric, 1, 4, mode="exact")
    try:
        r.set_early_stop(cfg)
        got = False
    except OverflowError:
        got = True
    assert got == raises
    try:
        orc.batch_query(c.graph, c.base, c.queries, 1, 4, metric=metric, early_stop=cfg)
        want = False
    except orc.EarlyStopNotRepresentable:
        want = True
    assert got == want
    r.close()


def test_thresholds_must_cover_every_upper_level():
    c = golden_case("early_stop_top2")
    r = GpuRouter(index_for(c.name), 1, 1, 4, mode="exact")
    with pytest.raises(ArteaGpuError):
        r.set_early_stop([0, 8])
    r.close()


def test_bottom_only_graph_accepts_any_thresholds():
    # test_router_early_stop.cpp:183-197.
    c = golden_case("early_stop_top0")
    r = GpuRouter(index_for(c.name), 1, 1, 4, mode="exact")
    r.set_early_stop([0, -1, np.nan])
    out = r.batch_query(c.queries[3:4])
    assert (int(out[0, 0]) & 0x7FFFFFFF) == 3
    r.close()


def test_cuda_graph_replay_follows_the_early_stop_setting():
    c = golden_case("sift2k")
    cfg, words, _ = c.es[1]
    L = c.queues[-1]
    r = GpuRouter(index_for("sift2k"), c.metric, c.topk, L, mode="exact", use_graphs=True)
    np.testing.assert_array_equal(r.batch_query(c.queries), c.words[L])
    np.testing.assert_array_equal(r.batch_query(c.queries), c.words[L])   # replayed
    r.set_early_stop(cfg)
    np.testing.assert_array_equal(r.batch_query(c.queries), words[L])
    np.testing.assert_array_equal(r.batch_query(c.queries), words[L])
    r.set_early_stop(None)
    np.testing.assert_array_equal(r.batch_query(c.queries), c.words[L])
    r.close()


class _Config:
    """Stands in for an RGraphConfig: early_stop_threshold(h, pruning)."""

    def __init__(self, thr):
        self.thr = thr
        self.evaluations = 0

    def early_stop_threshold(self, h, pruning):
        self.evaluations += 1
        return self.thr[h]


def test_drop_in_config_overload_evaluates_each_level_once():
    # test_router_early_stop.cpp:160-180: thresholds computed once per batch.
    c = golden_case("early_stop_top2")
    router = HierarchicalGraphRouter(c.base, "euclidean", topk=1, candidate_queue_size=4)
    router.initialize()
    cfg = _Config([0, 8, 16])
    words = router.batch_query(c.queries, c.graph, cfg, object(), enable_early_stop=True)
    assert cfg.evaluations == 2
    assert [int(w) & 0x7FFFFFFF for w in words] == [0, 1, 2, 3]
    np.testing.assert_array_equal(words.reshape(-1, 1), c.es[0][1][4])
    router.close()
