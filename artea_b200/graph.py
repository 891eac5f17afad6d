"""Host-side compact hierarchical graph (the reference's compact::HierarchicalGraph).

Mirrors index/compact_structure/hierarchical_graph.hpp:33-201: a vertex table
of (highest_level, local_vid), one CSR offset array per highest-level group
(group h has N_h*(h+1)+1 offsets, each vertex's rows from level h down to 0)
and one global neighbour-id array. Snapshots use the reference's HGRA v1
format (index/persistence/hierarchical_graph_file_manager.hpp:15-39), read and
written by the native library.
"""

from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence

import numpy as np

from . import _native as nat

INVALID_LEVEL = 0xFFFFFFFF
INVALID_VID = 0xFFFFFFFF


class CompactHierarchicalGraph:
    """Grouped-CSR graph held in numpy arrays (host memory)."""

    is_compacted = True
    invalid_level_id = INVALID_LEVEL

    def __init__(self, num_vertices: int, top_level: int, ul_max_nbr_size: int, bl_max_nbr_size: int,
                 entry_point_vid: int, vertex_info: np.ndarray, group_offsets: Sequence[np.ndarray],
                 neighbor_ids: np.ndarray):
        self.num_vertices = int(num_vertices)
        self.top_level = int(top_level)
        self.ul_max_nbr_size = int(ul_max_nbr_size)
        self.bl_max_nbr_size = int(bl_max_nbr_size)
        self.entry_point_vid = int(entry_point_vid)
        self.vertex_info = np.ascontiguousarray(vertex_info, dtype=np.uint32).reshape(-1, 2)
        self.group_offsets: List[np.ndarray] = [np.ascontiguousarray(o, dtype=np.uint64) for o in group_offsets]
        self.neighbor_ids = np.ascontiguousarray(neighbor_ids, dtype=np.uint32)
        self._desc_keepalive = None

    # ---- reference accessors -------------------------------------------------
    def get_num_vertices(self) -> int:
        return self.num_vertices

    def top_occupied_level_id(self) -> int:
        """hierarchical_graph.hpp:118-120: invalid for an empty graph."""
        return INVALID_LEVEL if self.num_vertices == 0 else self.top_level

    def entry_point(self) -> int:
        return self.entry_point_vid

    def group_sizes(self) -> np.ndarray:
        return np.array([(len(o) - 1) // (h + 1) for h, o in enumerate(self.group_offsets)], dtype=np.uint64)

    def fetch_level_nbrs(self, vid: int, level: int) -> np.ndarray:
        """hierarchical_graph.hpp:99-108."""
        hl, local = (int(x) for x in self.vertex_info[vid])
        row = local * (hl + 1) + (hl - level)
        off = self.group_offsets[hl]
        return self.neighbor_ids[int(off[row]):int(off[row + 1])]

    def level_histogram(self) -> List[int]:
        return [int(s) for s in self.group_sizes()]

    # ---- construction --------------------------------------------------------
    @classmethod
    def from_rows(cls, num_vertices: int, highest_level: Sequence[int], rows: Sequence[Sequence[Sequence[int]]],
                  entry_point_vid: int, ul_max_nbr_size: int = 32, bl_max_nbr_size: int = 64,
                  top_level: Optional[int] = None) -> "CompactHierarchicalGraph":
        """Build from per-vertex rows: rows[v][level] is the neighbour list of v
        at ``level`` (levels 0..highest_level[v]); highest_level[v] may be
        INVALID_LEVEL for an unassigned vertex. Local ids follow vid order,
        as the reference's restore assigns them."""
        hl = [int(h) for h in highest_level]
        top = max((h for h in hl if h != INVALID_LEVEL), default=0) if top_level is None else int(top_level)
        groups = top + 1
        buckets: List[List[int]] = [[] for _ in range(groups)]
        vinfo = np.full((num_vertices, 2), INVALID_VID, dtype=np.uint32)
        for v in range(num_vertices):
            if hl[v] == INVALID_LEVEL:
                continue
            vinfo[v] = (hl[v], len(buckets[hl[v]]))
            buckets[hl[v]].append(v)
        offsets = []
        nbrs: List[int] = []
        for h in range(groups):
            off = [len(nbrs)]
            for v in buckets[h]:
                for level in range(h, -1, -1):
                    nbrs.extend(int(x) for x in rows[v][level])
                    off.append(len(nbrs))
            offsets.append(np.array(off, dtype=np.uint64))
        return cls(num_vertices, top, ul_max_nbr_size, bl_max_nbr_size, entry_point_vid, vinfo, offsets,
                   np.array(nbrs, dtype=np.uint32))

    @classmethod
    def from_hgra(cls, path: str) -> "CompactHierarchicalGraph":
        """HierarchicalGraphFileManager::restore, via the native reader."""
        L = nat.lib()
        info = nat.HgraInfo()
        nat.check(L.artea_gpu_hgra_probe(os.fsencode(path), ctypes.byref(info)))
        vinfo = np.empty((info.num_vertices, 2), dtype=np.uint32)
        offsets = np.empty(max(info.num_offsets, 1), dtype=np.uint64)
        nbrs = np.empty(max(info.num_neighbor_ids, 1), dtype=np.uint32)
        nat.check(L.artea_gpu_hgra_read(os.fsencode(path), nat.ptr(vinfo), nat.ptr(offsets), nat.ptr(nbrs)))
        groups = []
        at = 0
        for h in range(info.num_groups):
            cnt = int(info.group_sizes[h]) * (h + 1) + 1
            groups.append(offsets[at:at + cnt])
            at += cnt
        return cls(info.num_vertices, info.top_level, info.ul_max_nbr_size, info.bl_max_nbr_size,
                   info.entry_point_vid, vinfo, groups, nbrs[: info.num_neighbor_ids])

    # ---- native description ----------------------------------------------------
    def desc(self) -> nat.GraphDesc:
        """A GraphDesc pointing at this graph's arrays (valid while self lives)."""
        groups = len(self.group_offsets)
        gptr = (ctypes.POINTER(ctypes.c_uint64) * max(groups, 1))()
        for h, o in enumerate(self.group_offsets):
            gptr[h] = o.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        sizes = np.ascontiguousarray(self.group_sizes(), dtype=np.uint64)
        if sizes.size == 0:
            sizes = np.zeros(1, dtype=np.uint64)
        d = nat.GraphDesc()
        d.num_vertices = self.num_vertices
        d.top_level = self.top_occupied_level_id()
        d.ul_max_nbr_size = self.ul_max_nbr_size
        d.bl_max_nbr_size = self.bl_max_nbr_size
        d.entry_point_vid = self.entry_point_vid
        d.vertex_info = self.vertex_info.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        d.group_offsets = ctypes.cast(gptr, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64)))
        d.group_sizes = sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        d.neighbor_ids = self.neighbor_ids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        d.num_neighbor_ids = int(self.neighbor_ids.size)
        self._desc_keepalive = (gptr, sizes)
        return d

    def validate(self) -> None:
        """Host validation the uploader applies (raises ArteaGpuError)."""
        d = self.desc()
        nat.check(nat.lib().artea_gpu_graph_validate(ctypes.byref(d)))

    def to_hgra(self, path: str) -> None:
        """HierarchicalGraphFileManager::snapshot."""
        d = self.desc()
        nat.check(nat.lib().artea_gpu_hgra_write(os.fsencode(path), ctypes.byref(d)))
