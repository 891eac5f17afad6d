"""artea_gpu_batch_query_noalloc: the batch query for callers that cannot
allocate device memory (inside an allocator callback, under a fully reserved
memory pool, in processes that forbid allocation after start-up). It takes
its scratch from a fixed device array instead of cudaMalloc. Its results must
equal the regular device entry point's (EXACT mode: bit for bit) on two calls
in a row, since every call reuses the array the previous call left behind."""
import numpy as np
import pytest

from conftest import golden_case
from artea_b200 import _native as nat
from artea_b200.router import DeviceIndex, GpuRouter

pytestmark = pytest.mark.gpu


def _run_noalloc(idx, metric, mode, k, L, d_q, nq, torch):
    out = torch.full((nq, k), -1, dtype=torch.int64, device=d_q.device)
    nat.check(nat.lib().artea_gpu_batch_query_noalloc(idx.handle, metric, mode, k, L, nat.ptr(d_q), nq, k,
                                                      nat.ptr(out), None))
    return out.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("name,L,mode", [("sift2k", 32, 0), ("sift2k", 100, 0), ("deep1k_cos", 64, 0),
                                         ("gist400", 50, 0), ("sift2k", 100, 1)])
def test_noalloc_matches_device_entry_point_on_consecutive_calls(name, L, mode):
    import torch
    c = golden_case(name)
    idx = DeviceIndex(c.graph, c.base)
    nq, k = c.queries.shape[0], c.topk
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    ref = torch.empty((nq, k), dtype=torch.int64, device=d_q.device)
    r = GpuRouter(idx, c.metric, k, L, mode="exact" if mode == 0 else "fast", schedule="persistent")
    r.batch_query_device(d_q, nq, k, ref)
    torch.cuda.synchronize()
    r.sync()
    expected = ref.cpu().numpy().view(np.uint64)
    if mode == 0:
        np.testing.assert_array_equal(expected, c.words[L])
    for _ in range(2):
        np.testing.assert_array_equal(_run_noalloc(idx, c.metric, mode, k, L, d_q, nq, torch), expected)
    r.close()
    idx.close()


def test_noalloc_rejects_out_of_limit_arguments():
    import torch
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    out = torch.empty((c.queries.shape[0], 10), dtype=torch.int64, device=d_q.device)
    L = nat.lib()
    assert L.artea_gpu_batch_query_noalloc(idx.handle, 0, 0, 10, 2048, nat.ptr(d_q), 4, 10, nat.ptr(out),
                                           None) == nat.EINVAL
    assert L.artea_gpu_batch_query_noalloc(idx.handle, 0, 0, 10, 5, nat.ptr(d_q), 4, 10, nat.ptr(out),
                                           None) == nat.EINVAL
    assert L.artea_gpu_batch_query_noalloc(idx.handle, 0, 0, 10, 32, None, 4, 10, nat.ptr(out), None) == nat.EINVAL
    idx.close()


def test_noalloc_call_leaves_device_free_memory_unchanged():
    # After a first call (which may load this library's module on the device,
    # and with it the scratch array), a later call must not take any device
    # memory: the free byte count the driver reports stays the same.
    import torch
    c = golden_case("sift2k")
    idx = DeviceIndex(c.graph, c.base)
    nq, k = c.queries.shape[0], c.topk
    d_q = torch.from_numpy(np.ascontiguousarray(c.queries)).cuda()
    out = torch.empty((nq, k), dtype=torch.int64, device=d_q.device)
    L = nat.lib()
    nat.check(L.artea_gpu_batch_query_noalloc(idx.handle, c.metric, 0, k, 32, nat.ptr(d_q), nq, k, nat.ptr(out), None))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        nat.check(L.artea_gpu_batch_query_noalloc(idx.handle, c.metric, 0, k, 32, nat.ptr(d_q), nq, k, nat.ptr(out),
                                                  None))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), c.words[32])
    idx.close()
