"""C-ABI library: loads, exports what include/artea_gpu.h declares, host-side
logic (HGRA snapshots, graph validation, argument checks) without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_case
from artea_b200 import _native as nat
from artea_b200.graph import CompactHierarchicalGraph, INVALID_LEVEL
from artea_b200.router import HierarchicalGraphRouter


def declared_functions():
    text = open(nat.HEADER_PATH).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(artea_gpu_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = nat.lib()
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(nat.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (artea_gpu_\w+)", out))
    assert set(names) <= exported


def test_library_built_for_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", nat.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_version_string():
    assert b"sm_100a" in nat.lib().artea_gpu_version()


def test_hgra_roundtrip_is_byte_identical(tmp_path):
    c = golden_case("sift2k")
    p = str(tmp_path / "rt.hgra")
    c.graph.to_hgra(p)
    assert open(p, "rb").read() == open(c.hgra_path, "rb").read()
    g2 = CompactHierarchicalGraph.from_hgra(p)
    np.testing.assert_array_equal(g2.vertex_info, c.graph.vertex_info)
    np.testing.assert_array_equal(g2.neighbor_ids, c.graph.neighbor_ids)
    for a, b in zip(g2.group_offsets, c.graph.group_offsets):
        np.testing.assert_array_equal(a, b)


def test_fetch_level_nbrs_matches_rows():
    c = golden_case("early_stop_top2")
    g = c.graph
    assert list(g.fetch_level_nbrs(0, 0)) == [1, 2, 3]
    assert list(g.fetch_level_nbrs(0, 1)) == [1]
    assert list(g.fetch_level_nbrs(2, 1)) == [3]
    assert list(g.fetch_level_nbrs(0, 2)) == []


def _status(fn):
    with pytest.raises(nat.ArteaGpuError) as e:
        fn()
    return e.value.status


def test_truncated_snapshot_is_rejected(tmp_path):
    c = golden_case("sift2k")
    data = open(c.hgra_path, "rb").read()
    p = tmp_path / "trunc.hgra"
    p.write_bytes(data[: len(data) // 2])
    assert _status(lambda: CompactHierarchicalGraph.from_hgra(str(p))) == nat.EIO
    p.write_bytes(b"XXXX" + data[4:])
    assert _status(lambda: CompactHierarchicalGraph.from_hgra(str(p))) == nat.EIO
    assert _status(lambda: CompactHierarchicalGraph.from_hgra(str(tmp_path / "missing.hgra"))) == nat.EIO


def _tiny(rows0, hl=None, entry=0):
    n = len(rows0)
    hl = hl or [0] * n
    rows = [{0: r} for r in rows0]
    return CompactHierarchicalGraph.from_rows(n, hl, rows, entry_point_vid=entry, ul_max_nbr_size=8, bl_max_nbr_size=8)


def test_validator_rejects_out_of_range_ids():
    g = _tiny([[1], [0, 5]])
    assert _status(g.validate) == nat.EGRAPH


def test_validator_rejects_bad_entry_point():
    g = _tiny([[1], [0]], entry=7)
    assert _status(g.validate) == nat.EGRAPH


def test_validator_rejects_rows_naming_vertices_absent_from_the_level():
    # vid 2 is only on L0 but appears in vid 0's L1 row.
    rows = [{0: [1, 2], 1: [1, 2]}, {0: [0], 1: [0]}, {0: [0]}]
    g = CompactHierarchicalGraph.from_rows(3, [1, 1, 0], rows, entry_point_vid=0, ul_max_nbr_size=8, bl_max_nbr_size=8)
    assert _status(g.validate) == nat.EGRAPH


def test_validator_rejects_overlong_rows():
    g = _tiny([[1] * 9, [0]])
    assert _status(g.validate) == nat.EGRAPH


def test_validator_accepts_reference_graphs():
    for name in ("early_stop_top0", "early_stop_top2", "axis80", "sift2k", "deep1k_cos", "gist400"):
        golden_case(name).graph.validate()


def test_empty_graph_validates_and_snapshots(tmp_path):
    g = CompactHierarchicalGraph(0, 0, 4, 4, INVALID_LEVEL & 0xFFFFFFFF, np.zeros((0, 2), np.uint32),
                                 [np.zeros(1, np.uint64)], np.zeros(0, np.uint32))
    g.validate()
    p = str(tmp_path / "empty.hgra")
    g.to_hgra(p)
    g2 = CompactHierarchicalGraph.from_hgra(p)
    assert g2.num_vertices == 0


def test_router_rejects_queue_smaller_than_topk():
    # hierarchical_graph_router.hpp:104-108 throws std::runtime_error.
    with pytest.raises(RuntimeError):
        HierarchicalGraphRouter(np.zeros((4, 16), np.float32), "euclidean_sqr", topk=10, candidate_queue_size=5)


def test_index_create_rejects_bad_dim_without_touching_the_gpu():
    c = golden_case("early_stop_top2")
    d = c.graph.desc()
    h = ctypes.c_void_p()
    base = np.zeros((4, 15), np.float32)
    rc = nat.lib().artea_gpu_index_create(ctypes.byref(d), nat.ptr(base), 4, 15, 0, ctypes.byref(h))
    assert rc == nat.EINVAL


def test_null_arguments_are_rejected():
    L = nat.lib()
    assert L.artea_gpu_hgra_probe(None, None) == nat.EINVAL
    assert L.artea_gpu_router_destroy(None) == nat.OK
    assert L.artea_gpu_index_destroy(None) == nat.OK
    assert L.artea_gpu_batch_query(None, None, 0, None, None, 0, None, None) == nat.EINVAL


def test_serving_percentiles_use_the_reference_profilers_pick():
    # hg_router_profiler.hpp:429-444: sorted[floor(n * p)], clamped; no interpolation.
    from artea_b200.serving import latency_percentile
    lat = [5.0, 1.0, 4.0, 2.0, 3.0]
    assert latency_percentile(lat, 0.50) == 3.0       # index 2
    assert latency_percentile(lat, 0.90) == 5.0       # index 4
    assert latency_percentile(lat, 0.99) == 5.0
    assert latency_percentile(list(range(100)), 0.99) == 99.0
    assert latency_percentile(list(range(100)), 0.95) == 95.0
    assert latency_percentile([7.0], 0.5) == 7.0
    assert np.isnan(latency_percentile([], 0.5))


def test_device_restore_rejects_bad_headers_before_touching_the_gpu(tmp_path):
    # artea_gpu_index_create_from_hgra checks the header (and the room for one
    # record per vertex) before it needs a device: the reader's EIO.
    import struct
    from artea_b200.router import DeviceIndex
    base = np.zeros((4, 16), np.float32)
    good = struct.pack("<7I", 0x48475241, 1, 2, 0, 4, 4, 0) + struct.pack("<6I", 0, 1, 1, 0, 1, 0)
    cases = {
        "short": good[:20],
        "misaligned": good + b"\x00",
        "magic": b"XXXX" + good[4:],
        "version": good[:4] + struct.pack("<I", 9) + good[8:],
        "top_none": good[:12] + struct.pack("<I", 0xFFFFFFFF) + good[16:],
        "top_64": good[:12] + struct.pack("<I", 64) + good[16:],
        "entry_range": good[:24] + struct.pack("<I", 5) + good[28:],
        "no_room": struct.pack("<7I", 0x48475241, 1, 9, 0, 4, 4, 0) + struct.pack("<2I", 0, 0),
        "empty_trailing": struct.pack("<7I", 0x48475241, 1, 0, 0, 4, 4, 0xFFFFFFFF) + struct.pack("<I", 0),
    }
    for name, data in cases.items():
        p = tmp_path / f"{name}.hgra"
        p.write_bytes(data)
        assert _status(lambda: DeviceIndex.from_hgra(str(p), base)) == nat.EIO, name
        assert _status(lambda: CompactHierarchicalGraph.from_hgra(str(p))) == nat.EIO, name
    assert _status(lambda: DeviceIndex.from_hgra(str(tmp_path / "missing.hgra"), base)) == nat.EIO
