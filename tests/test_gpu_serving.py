"""Serving loop (continuous batching): each request's result is the same
whether it runs alone or mixed with others in flight (EXACT mode: bit for
bit, and equal to the oracle); admission follows the ring's free slots; the
resident kernel ends once the host heartbeat goes stale (failure injected on
the host), freeing the GPU, and unfinished work then reports ETIMEOUT. Every
server is closed by a with block, so a failing assertion cannot leave a
resident kernel behind for the next test."""
import threading
import time

import numpy as np
import pytest

from conftest import golden_case
from artea_b200 import _native as nat
from artea_b200.router import DeviceIndex, GpuRouter
from artea_b200.serving import Server, make_requests, run_poisson
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _expected(c, lo, n, topk, queue, k_stride):
    return orc.batch_query(c.graph, c.base, c.queries[lo:lo + n], topk, queue, metric=c.metric, k_stride=k_stride)


@pytest.mark.parametrize("name", ["sift2k", "deep1k_cos"])
def test_results_alone_equal_results_in_the_mix(name):
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    with Server(idx, c.metric, max_topk=10, max_queue=100, ring_slots=256) as srv:
        _alone_and_mixed(c, srv)


def _alone_and_mixed(c, srv):
    nq = c.queries.shape[0]
    rng = np.random.default_rng(5)
    sizes, reqs, lo = [], [], 0
    while lo < nq:
        n = int(min(nq - lo, rng.integers(1, 12)))
        k = np.full(n, int(rng.choice([1, 5, 10])), np.uint32)
        L = np.maximum(np.full(n, int(rng.choice([10, 32, 100])), np.uint32), k)
        reqs.append((lo, n, k, L))
        lo += n
    # alone: one request at a time on an otherwise idle server
    alone = []
    for lo, n, k, L in reqs:
        t = srv.submit(c.queries[lo:lo + n], k, L)
        alone.append(srv.wait(t, n, 10))
    # in the mix: everything submitted before anything is polled
    tickets = [srv.submit(c.queries[lo:lo + n], k, L) for lo, n, k, L in reqs]
    mixed = [srv.wait(t, n, 10) for t, (lo, n, k, L) in zip(tickets, reqs)]
    for (lo, n, k, L), a, m in zip(reqs, alone, mixed):
        np.testing.assert_array_equal(a, m)
        np.testing.assert_array_equal(a, _expected(c, lo, n, k, L, 10))


def test_admission_by_ring_slots():
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    with Server(idx, 0, max_topk=10, max_queue=32, ring_slots=8) as srv:
        with pytest.raises(nat.ArteaGpuError):
            srv.submit(c.queries[:9])                      # larger than the ring
        t1 = srv.submit(c.queries[:5])
        assert srv.submit(c.queries[5:10]) is None          # 5 + 5 > 8 slots in flight
        r1 = srv.wait(t1, 5, 10)
        t2 = srv.submit(c.queries[5:10])                    # admitted once slots are freed
        r2 = srv.wait(t2, 5, 10)
        np.testing.assert_array_equal(np.vstack([r1, r2]), c.words[32][:10])


def test_idle_exit_is_refused():
    # An idle exit followed by a relaunch on the same stream was seen to leave
    # the new kernel unstarted; the option is refused until that is explained.
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    with pytest.raises(nat.ArteaGpuError) as e:
        Server(idx, 0, max_topk=10, max_queue=32, ring_slots=64, idle_polls=20)
    assert e.value.status == nat.EINVAL


def test_stale_heartbeat_ends_the_kernel_and_reports_timeout():
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    with Server(idx, 0, max_topk=10, max_queue=32, ring_slots=64, heartbeat_ms=300) as srv:
        r1 = srv.wait(srv.submit(c.queries[:8]), 8, 10)
        time.sleep(1.0)                                  # idle for 3 limits, heartbeat alive: still resident
        r2 = srv.wait(srv.submit(c.queries[8:16]), 8, 10, timeout_s=10)
        np.testing.assert_array_equal(np.vstack([r1, r2]), c.words[32][:16])
        assert srv.stats()["kernel_launches"] == 1
        srv.pause_heartbeat()                            # the host stops answering
        # A batch query of another router can only run once the resident kernel
        # has left the SMs; it must finish soon after the limit passes.
        router = GpuRouter(idx, 0, 10, 32, schedule="plain")
        out = {}

        def other():
            out["words"] = router.batch_query(c.queries[:16])

        th = threading.Thread(target=other)
        th.start()
        th.join(timeout=10.0)
        left = not th.is_alive()
        if not left:
            srv.close()                                  # stop flag: releases the kernel, then fail
            th.join(timeout=30.0)
        assert left, "the serving kernel did not end after its heartbeat went stale"
        np.testing.assert_array_equal(out["words"], c.words[32][:16])
        with pytest.raises(nat.ArteaGpuError) as e:
            srv.submit(c.queries[16:20])
        assert e.value.status == nat.ETIMEOUT
        router.close()


def test_poisson_load_results_match_oracle():
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    qs = np.vstack([c.queries] * 8)
    reqs = make_requests(qs.shape[0], rate_qps=20000, seed=3, topk_choices=(5, 10), queue_choices=(32, 100),
                         max_size=32)
    with Server(idx, 0, max_topk=10, max_queue=100, ring_slots=512) as srv:
        stats = run_poisson(srv, qs, reqs, 10, timeout_s=60)
    assert stats["queries"] == qs.shape[0]
    for r in reqs:
        exp = orc.batch_query(c.graph, c.base, qs[r.lo:r.lo + r.n], r.topk, r.queue, metric=0, k_stride=10)
        np.testing.assert_array_equal(r.result, exp)
