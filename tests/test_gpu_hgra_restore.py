"""HGRA snapshot restored straight to the device (artea_gpu_index_create_from_hgra)
against the host reader + upload (artea_gpu_hgra_read + artea_gpu_index_create):
the same device graph word for word, the same search results, and the same
status on every damaged file the host path rejects."""
import struct

import numpy as np
import pytest

from conftest import big_snapshot, golden_case
from artea_b200 import _native as nat
from artea_b200.graph import CompactHierarchicalGraph
from artea_b200.router import DeviceIndex, GpuRouter

pytestmark = pytest.mark.gpu

MAGIC, VERSION, NONE = 0x48475241, 1, 0xFFFFFFFF


def host_arrays(g: CompactHierarchicalGraph):
    offs = np.concatenate(g.group_offsets) if g.group_offsets else np.zeros(0, np.uint64)
    return g.vertex_info, offs, g.neighbor_ids


def assert_same_device_graph(path, base):
    g = CompactHierarchicalGraph.from_hgra(path)
    ix = DeviceIndex.from_hgra(path, base)
    vi, offs, nb = host_arrays(g)
    got = ix.download_graph(g.num_vertices, offs.size, nb.size)
    np.testing.assert_array_equal(got[0], vi)
    np.testing.assert_array_equal(got[1], offs)
    np.testing.assert_array_equal(got[2], nb)
    ref = DeviceIndex(g, base)
    assert ix.nbytes() == ref.nbytes()
    ref.close()
    return ix


@pytest.mark.parametrize("name", ["early_stop_top2", "axis80", "sift2k", "deep1k_cos", "gist400"])
def test_restored_graph_and_results_equal_the_host_path(name):
    c = golden_case(name)
    ix = assert_same_device_graph(c.hgra_path, c.base)
    for L in c.queues:
        r = GpuRouter(ix, c.metric, c.topk, L, mode="exact")
        np.testing.assert_array_equal(r.batch_query(c.queries), c.words[L], err_msg=f"{name} L={L}")
        r.close()
    ix.close()


def write_hgra(path, n, top, ul, bl, entry, records):
    """records: per vid, None (unassigned) or a list of rows from the highest level down to 0."""
    words = [MAGIC, VERSION, n, top, ul, bl, entry]
    for rows in records:
        if rows is None:
            words.append(NONE)
            continue
        words.append(len(rows) - 1)
        for r in rows:
            words.append(len(r))
            words.extend(r)
    with open(path, "wb") as f:
        f.write(struct.pack(f"<{len(words)}I", *words))


def test_records_straddling_the_staging_chunks(tmp_path):
    path = str(tmp_path / "big.hgra")
    base = big_snapshot(path)
    ix = assert_same_device_graph(path, base)
    ix.close()


def _status(fn):
    try:
        ix = fn()
    except nat.ArteaGpuError as e:
        return e.status
    ix.close()
    return nat.OK


def host_path(path, base):
    return DeviceIndex(CompactHierarchicalGraph.from_hgra(path), base)


@pytest.mark.parametrize("case", [
    "ok", "id_out_of_range", "off_level", "entry_not_top", "entry_none", "row_over_capacity", "upper_over_capacity",
    "above_top", "trailing", "truncated_row", "truncated_vid", "truncated_count", "bad_magic", "bad_version",
    "unassigned_vertex", "empty",
])
def test_damaged_snapshots_get_the_host_paths_status(tmp_path, case):
    p = str(tmp_path / f"{case}.hgra")
    n, top, ul, bl, entry, recs = 3, 1, 4, 4, 0, [[[1], [1, 2]], [[0], [0]], [[0]]]
    raw = None
    if case == "id_out_of_range":
        recs = [[[1], [1, 7]], [[0], [0]], [[0]]]
    elif case == "off_level":
        recs = [[[2], [1, 2]], [[0], [0]], [[0]]]        # vid 2 is only on level 0
    elif case == "entry_not_top":
        entry = 2
    elif case == "entry_none":
        entry = NONE
    elif case == "row_over_capacity":
        recs = [[[1], [1, 2, 1, 2, 1]], [[0], [0]], [[0]]]
    elif case == "upper_over_capacity":
        ul = 0
    elif case == "above_top":
        recs = [[[1], [1, 2]], [[0], [0]], [[0], [0], [0]]]
    elif case == "unassigned_vertex":
        recs = [[[1], [1]], [[0], [0]], None]
    elif case == "empty":
        n, top, entry, recs = 0, 0, NONE, []
    write_hgra(p, n, top, ul, bl, entry, recs)
    data = open(p, "rb").read()
    if case == "trailing":
        raw = data + struct.pack("<I", 5)
    elif case == "truncated_row":
        raw = data[:-4]
    elif case == "truncated_vid":
        raw = data[:-8]                                   # vid 2's record cut after its level word
    elif case == "truncated_count":
        raw = data[: 4 * (7 + 1 + 1 + 1 + 1 + 2 + 1)]     # cut before vid 1's first count
    elif case == "bad_magic":
        raw = b"XXXX" + data[4:]
    elif case == "bad_version":
        raw = data[:4] + struct.pack("<I", 2) + data[8:]
    if raw is not None:
        open(p, "wb").write(raw)
    base = np.zeros((max(n, 1), 16), np.float32)
    want = _status(lambda: host_path(p, base))
    got = _status(lambda: DeviceIndex.from_hgra(p, base))
    assert got == want, f"{case}: device path {got}, host path {want}"
    if case == "ok":
        assert got == nat.OK
    if case == "empty":
        ix = DeviceIndex.from_hgra(p, base)
        r = GpuRouter(ix, 0, 2, 4, mode="exact")
        out = r.batch_query(np.zeros((2, 16), np.float32))
        assert (out == np.uint64((0x7F7FFFFF << 32) | 0x7FFFFFFF)).all()
        r.close()
        ix.close()


def test_download_needs_a_graph():
    from artea_b200.router import vectors_only_graph
    ix = DeviceIndex(vectors_only_graph(), np.zeros((4, 16), np.float32))
    with pytest.raises(nat.ArteaGpuError):
        ix.download_graph(0, 1, 0)
    ix.close()
