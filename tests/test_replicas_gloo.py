"""N>1 host path (replicas): 2 gloo ranks on CPU split a batch, search their
shard with the oracle standing in for the per-GPU router, and all-gather the
rows; the result must equal one process answering the whole batch."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT, golden_case
from artea_b200.replicas import shard


def test_shards_cover_the_batch():
    for nq in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard(nq, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nq
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    from conftest import golden_case as gc
    from artea_b200.replicas import ReplicatedRouter
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    c = gc("sift2k")
    router = ReplicatedRouter(lambda q: orc.batch_query(c.graph, c.base, q, 10, 32, metric=0, threads=2), 10)
    res = router.batch_query(c.queries)
    if rank == 0:
        np.save(out_path, res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_process(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    res = np.load(out)
    c = golden_case("sift2k")
    np.testing.assert_array_equal(res, c.words[32])
