"""Config 0 at its stated size: 100,000 x 128 integer-valued vectors (256-centre
mixture), the graph built by the reference builder with beta 2.0, tau_k 0,
tau 1.5, l0_min_distance 1.0, search_nn_qs 64, 15 loops, 4 triu iterations,
prefill 0.4, pruning scale 1.10 / shift 1.5, shuffle; 1,000 queries from the
same mixture, topk 100, queue 200, RandomSeeding=false.

EXACT mode must return the reference router's words bit for bit (its own
batch_query compiled from its headers where the host can run it, else the C
restatement), on every schedule and level-0 loop, and inherit its recall."""
import numpy as np
import pytest

from artea_b200 import workload as wl
from artea_b200.graph import CompactHierarchicalGraph
from artea_b200.router import DeviceIndex, GpuRouter
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOPK, QUEUE = 100, 200


def _host_has_avx512() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f in flags for f in ("avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd"))


@pytest.fixture(scope="module")
def config0():
    try:
        w, base, queries, hgra, report = wl.prepare("sift100k")
    except FileNotFoundError as e:
        pytest.skip(str(e))
    assert base.shape == (100_000, 128) and queries.shape == (1_000, 128)
    g = CompactHierarchicalGraph.from_hgra(hgra)
    if orc.have_ref() and _host_has_avx512():
        r = orc.RefRouter(hgra, base)
        ref, _ = r.batch_query(queries, TOPK, QUEUE, metric=0)
        r.close()
    else:
        ref = orc.batch_query(g, base, queries, TOPK, QUEUE, metric=0)
    idx = DeviceIndex(g, base)
    yield g, base, queries, ref, idx
    idx.close()


@pytest.mark.parametrize("schedule,pipeline", [("persistent", 0), ("persistent", 0xFFFFFFFF), ("plain", 0)])
def test_config0_exact_words_equal_reference(config0, schedule, pipeline):
    g, base, queries, ref, idx = config0
    r = GpuRouter(idx, 0, TOPK, QUEUE, mode="exact", schedule=schedule, pipeline=pipeline, max_batch=1000)
    out = r.batch_query(queries)
    bad = np.nonzero(~np.all(out == ref, axis=1))[0]
    assert bad.size == 0, f"{bad.size} of 1000 rows differ, first {bad[:5]}"
    r.close()


def test_config0_recall_is_the_references(config0):
    g, base, queries, ref, idx = config0
    words = idx.bruteforce(queries, TOPK, 0)
    gt = (words & np.uint64(0x7FFFFFFF)).astype(np.uint32)
    r = GpuRouter(idx, 0, TOPK, QUEUE, mode="exact")
    out = r.batch_query(queries)
    assert orc.recall_at_k(out, gt, TOPK) == orc.recall_at_k(ref, gt, TOPK)
    assert orc.recall_at_k(out, gt, TOPK) > 0.95
    r.close()
