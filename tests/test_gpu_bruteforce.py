"""GPU brute force (artea_gpu_bruteforce) against the reference's
bruteforce_router_t outputs and the oracle: distance bits identical, ids
identical up to the order of equal distances, CandidateEntry() padding."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_same_knn, golden_case
from artea_b200 import datasets as ds
from artea_b200._native import ArteaGpuError
from artea_b200.router import BruteforceRouter, DeviceIndex, vectors_only_graph
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [("early_stop_top2", [1, 3, 10]), ("axis80", [10, 100]), ("sift2k", [10, 100]), ("deep1k_cos", [10, 64]),
         ("gist400", [10, 50])]
PAD = np.uint64(0xFFFFFFFF)


@pytest.mark.parametrize("name,topks", CASES)
def test_bruteforce_matches_reference(name, topks):
    c = golden_case(name)
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    idx = DeviceIndex(c.graph, c.base)
    for k in topks:
        got = idx.bruteforce(c.queries, k, c.metric)
        assert_same_knn(got, z[f"bf_k{k}"], f"{name} k={k}")
        sub = z["bf_subset"]
        got = idx.bruteforce(c.queries, k, c.metric, subset=sub)
        assert_same_knn(got, z[f"bf_sub_k{k}"], f"{name} subset k={k}")
    idx.close()


def _data(metric, n, nq, seed):
    if metric == 2:
        w = ds.WORKLOADS["deep10m"].scaled(n, nq)
    else:
        w = ds.WORKLOADS["sift100k"].scaled(n, nq)
    base, queries = ds.generate(w)
    if metric == 3:
        rng = np.random.default_rng(seed)
        base = rng.standard_normal(base.shape).astype(np.float32)
        queries = rng.standard_normal(queries.shape).astype(np.float32)
    return base, queries


@pytest.mark.parametrize("metric", [0, 1, 2, 3])
@pytest.mark.parametrize("n,topk", [(5000, 100), (20000, 10), (20000, 1024)])
def test_bruteforce_matches_oracle(metric, n, topk):
    # 20000 rows split into several segments (merge kernel); 5000 rows in one.
    base, queries = _data(metric, n, 45, seed=n + topk)
    idx = DeviceIndex(vectors_only_graph(), base)
    got = idx.bruteforce(queries, topk, metric)
    ids, d = orc.bruteforce(base, queries, topk, metric=metric)
    want = (d.view(np.uint32).astype(np.uint64) << np.uint64(32)) | ids.astype(np.uint64)
    assert_same_knn(got, want, f"metric={metric} n={n} k={topk}")
    idx.close()


def test_bruteforce_padding_and_limits():
    base, queries = _data(0, 300, 9, seed=1)
    idx = DeviceIndex(vectors_only_graph(), base)
    got = idx.bruteforce(queries, 500, 0)                      # more than the rows
    assert (got[:, 300:] == PAD).all()
    ids, d = orc.bruteforce(base, queries, 300, metric=0)
    want = (d.view(np.uint32).astype(np.uint64) << np.uint64(32)) | ids.astype(np.uint64)
    assert_same_knn(got[:, :300], want, "all rows")
    assert (idx.bruteforce(queries, 7, 0, subset=np.zeros(0, np.uint32)) == PAD).all()
    for bad in (0, 1025):
        with pytest.raises(ArteaGpuError):
            idx.bruteforce(queries, bad, 0)
    with pytest.raises(ArteaGpuError):
        idx.bruteforce(queries, 5, 0, subset=np.array([0, 300], np.uint32))
    idx.close()


def test_bruteforce_device_entry_point_matches_host_one():
    import torch
    base, queries = _data(2, 6000, 17, seed=3)
    idx = DeviceIndex(vectors_only_graph(), base)
    host = idx.bruteforce(queries, 64, 2)
    dq = torch.from_numpy(queries).cuda()
    dout = torch.empty((17, 64), dtype=torch.int64, device="cuda")
    idx.bruteforce_device(dq, 17, 64, 2, dout)
    np.testing.assert_array_equal(dout.cpu().numpy().view(np.uint64), host)
    idx.close()


def test_bruteforce_router_surface():
    # bruteforce_router.hpp:74-96 query returns min(topk, n) entries; batch rows pad.
    c = golden_case("early_stop_top2")
    z = np.load(os.path.join(GOLDEN, "early_stop_top2.npz"))
    r = BruteforceRouter(c.base, "euclidean", topk=10)
    r.initialize()
    one = r.query(c.queries[2])
    assert one.size == 4
    assert_same_knn(r.batch_query(c.queries).reshape(-1, 10), z["bf_k10"], "batch")
    assert_same_knn(one.reshape(1, -1), z["bf_k10"][2][:4].reshape(1, -1), "query")
    r.close()


@pytest.mark.parametrize("name,metric", [("sift2k", 1), ("deep1k_cos", 2), ("gist400", 1)])
def test_centroid_entry_matches_the_reference_compactor(name, metric):
    # hierarchical_graph_compactor.hpp:236-248 chose each graph's entry point.
    c = golden_case(name)
    top = c.graph.top_occupied_level_id()
    bucket = np.nonzero(c.graph.vertex_info[:, 0] == top)[0].astype(np.uint32)
    idx = DeviceIndex(c.graph, c.base)
    assert idx.centroid_entry(metric, bucket) == c.graph.entry_point_vid
    assert idx.centroid_entry(metric, np.zeros(0, np.uint32)) == 0xFFFFFFFF
    idx.close()


def test_centroid_entry_matches_oracle_on_many_rows():
    for metric in (0, 1, 2, 3):
        base, _ = _data(metric, 30000, 1, seed=11)
        idx = DeviceIndex(vectors_only_graph(), base)
        assert idx.centroid_entry(metric) == orc.centroid_entry(base, metric)
        sub = np.arange(5, 30000, 7, dtype=np.uint32)
        assert idx.centroid_entry(metric, sub) == orc.centroid_entry(base, metric, sub)
        idx.close()
