"""The C++ drop-in: artea::cuda::HierarchicalGraphRouter<RouterTraitsT>
(include/artea_b200/hierarchical_graph_router.hpp) against the reference's
CPU hierarchical_graph_router_t on the reference's own compact graph type,
driven by tests/cpp/test_dropin.cpp."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden_case
from artea_b200 import datasets as ds

BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_dropin")


def _need_bin():
    if not os.path.exists(BIN):
        pytest.skip("drop-in check not built (needs the reference headers at build time)")


def test_dropin_constructor_contract():
    _need_bin()
    out = subprocess.run([BIN, "--cpu-only"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "OK constructor contract" in out.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name,topk,L", [("sift2k", 10, 32), ("sift2k", 10, 100), ("deep1k_cos", 10, 64),
                                         ("gist400", 10, 50), ("early_stop_top2", 1, 4), ("axis80", 10, 16)])
def test_dropin_matches_reference_router(name, topk, L):
    _need_bin()
    c = golden_case(name)
    with tempfile.TemporaryDirectory() as tmp:
        b, q = os.path.join(tmp, "b.fbin"), os.path.join(tmp, "q.fbin")
        ds.write_fbin(b, c.base.astype(np.float32))
        ds.write_fbin(q, c.queries.astype(np.float32))
        out = subprocess.run([BIN, c.hgra_path, b, q, str(c.metric), str(topk), str(L)], capture_output=True,
                             text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
