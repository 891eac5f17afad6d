"""ORACLE — test infrastructure only.

ctypes bindings of the two checkers:
  * ``liboracle.so`` — the plain-C restatement of the reference query path
    (artea_oracle.c), which travels with the tree and runs anywhere;
  * ``libartea_ref.so`` — the reference's own CPU router compiled from the
    reference headers (ref_bridge.cpp), present where it was built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm import
this module, and only as the checker.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libartea_ref.so")

INVALID_WORD = np.uint64((0x7F7FFFFF << 32) | 0x7FFFFFFF)
STATS_FIELDS = ("dist_evals", "upper_rows", "upper_row_ids", "l0_rows", "l0_row_ids", "upper_dist_evals",
                "results", "reserved")


class _Graph(ctypes.Structure):
    _fields_ = [
        ("num_vertices", c_uint32),
        ("top_level", c_uint32),
        ("entry_point", c_uint32),
        ("vinfo", POINTER(c_uint32)),
        ("offsets", POINTER(POINTER(c_uint64))),
        ("nbrs", POINTER(c_uint32)),
    ]


_olib = None
_rlib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        L = ctypes.CDLL(ORACLE_LIB)
        L.oracle_distance.restype = c_float
        L.oracle_distance.argtypes = [c_int, c_void_p, c_void_p, c_uint32]
        L.oracle_batch_query.restype = c_int
        L.oracle_batch_query.argtypes = [POINTER(_Graph), c_void_p, c_uint32, c_void_p, c_uint32, c_void_p, c_void_p,
                                         c_uint32, c_int, c_int, c_void_p, c_void_p, c_int]
        L.oracle_batch_query_early_stop.restype = c_int
        L.oracle_batch_query_early_stop.argtypes = [POINTER(_Graph), c_void_p, c_uint32, c_void_p, c_uint32, c_void_p,
                                                    c_void_p, c_uint32, c_int, c_void_p, c_uint32, c_void_p, c_void_p,
                                                    c_int]
        L.oracle_centroid_entry.restype = c_uint32
        L.oracle_centroid_entry.argtypes = [c_void_p, c_uint32, c_void_p, c_uint32, c_int]
        L.oracle_bruteforce.restype = c_int
        L.oracle_bruteforce.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p, c_uint32, c_uint32, c_int, c_void_p,
                                        c_void_p, c_int]
        _olib = L
    return _olib


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _rlib
    if _rlib is None:
        if not have_ref():
            raise ImportError(f"{REF_LIB} missing: run `make -C oracle` where the reference is mounted")
        L = ctypes.CDLL(REF_LIB)
        L.artea_ref_last_error.restype = c_char_p
        L.artea_ref_open.restype = c_void_p
        L.artea_ref_open.argtypes = [c_char_p, c_void_p, c_uint32, c_uint32]
        L.artea_ref_close.argtypes = [c_void_p]
        L.artea_ref_batch_query.restype = c_int
        L.artea_ref_batch_query.argtypes = [c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_int, c_int, c_int,
                                            c_void_p, POINTER(c_double), c_void_p]
        L.artea_ref_batch_query_early_stop.restype = c_int
        L.artea_ref_batch_query_early_stop.argtypes = [c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_int,
                                                       c_void_p, c_uint32, c_void_p, c_void_p]
        L.artea_ref_bruteforce.restype = c_int
        L.artea_ref_bruteforce.argtypes = [c_void_p, c_void_p, c_uint32, c_uint32, c_int, c_void_p, c_uint32,
                                           c_void_p]
        L.artea_ref_distance.restype = c_float
        L.artea_ref_distance.argtypes = [c_int, c_void_p, c_void_p, c_uint32]
        L.artea_ref_max_threads.restype = c_int
        L.artea_ref_restore_layout.restype = c_int
        L.artea_ref_restore_layout.argtypes = [c_char_p, c_void_p, c_void_p, c_void_p, c_void_p]
        L.artea_ref_restore_seconds.restype = ctypes.c_longlong
        L.artea_ref_restore_seconds.argtypes = [c_char_p, POINTER(c_double)]
        _rlib = L
    return _rlib


def _p(a):
    return c_void_p(None) if a is None else c_void_p(a.ctypes.data)


def distance(metric: int, a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return float(oracle_lib().oracle_distance(metric, _p(a), _p(b), a.size))


def ref_distance(metric: int, a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return float(ref_lib().artea_ref_distance(metric, _p(a), _p(b), a.size))


def ref_restore_layout(hgra_path: str):
    """The reference's HierarchicalGraphFileManager::restore of a snapshot as
    (vertex_info (n, 2) uint32, offsets of all groups concatenated uint64,
    neighbour ids uint32)."""
    L = ref_lib()
    sizes = np.zeros(4, dtype=np.uint64)
    p = os.fsencode(hgra_path)
    if L.artea_ref_restore_layout(p, _p(sizes), None, None, None) != 0:
        raise RuntimeError(L.artea_ref_last_error().decode())
    n, _, total, ids = (int(x) for x in sizes)
    vinfo = np.empty((n, 2), dtype=np.uint32)
    offs = np.empty(max(total, 1), dtype=np.uint64)
    nbrs = np.empty(max(ids, 1), dtype=np.uint32)
    if L.artea_ref_restore_layout(p, _p(sizes), _p(vinfo), _p(offs), _p(nbrs)) != 0:
        raise RuntimeError(L.artea_ref_last_error().decode())
    return vinfo, offs[:total], nbrs[:ids]


def ref_restore_seconds(hgra_path: str) -> float:
    """The reference's HierarchicalGraphFileManager::restore of a snapshot, timed."""
    secs = c_double()
    n = ref_lib().artea_ref_restore_seconds(os.fsencode(hgra_path), ctypes.byref(secs))
    if n < 0:
        raise RuntimeError(ref_lib().artea_ref_last_error().decode())
    return secs.value


class EarlyStopNotRepresentable(OverflowError):
    """The reference's std::overflow_error from _early_stop_thresholds."""


def batch_query(graph, base: np.ndarray, queries: np.ndarray, topk, queue, metric: int = 0, l0_only: bool = False,
                k_stride: int = None, threads: int = None, stats: bool = False, early_stop=None):
    """C restatement of batch_query; graph is an artea_b200.graph.CompactHierarchicalGraph.

    topk/queue: ints or per-query arrays. early_stop: per-level configuration
    thresholds (index = level) for enable_early_stop=true, or None. Returns
    (nq, k_stride) uint64 words and, if stats, an (nq, 8) uint32 counter array."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq = q.shape[0]
    tk = np.broadcast_to(np.asarray(topk, dtype=np.uint32), (nq,)).copy()
    qu = np.broadcast_to(np.asarray(queue, dtype=np.uint32), (nq,)).copy()
    if k_stride is None:
        k_stride = int(tk.max()) if nq else 0
    out = np.empty((nq, k_stride), dtype=np.uint64)
    st = np.zeros((nq, 8), dtype=np.uint32) if stats else None
    offs = (POINTER(c_uint64) * max(len(graph.group_offsets), 1))()
    for h, o in enumerate(graph.group_offsets):
        offs[h] = o.ctypes.data_as(POINTER(c_uint64))
    g = _Graph(graph.num_vertices, graph.top_occupied_level_id(), graph.entry_point_vid,
               graph.vertex_info.ctypes.data_as(POINTER(c_uint32)),
               ctypes.cast(offs, POINTER(POINTER(c_uint64))),
               graph.neighbor_ids.ctypes.data_as(POINTER(c_uint32)))
    threads = threads or os.cpu_count() or 1
    if early_stop is not None:
        if l0_only:
            raise ValueError("early stop applies to the hierarchical query only")
        thr = np.ascontiguousarray(early_stop, dtype=np.float32)
        rc = oracle_lib().oracle_batch_query_early_stop(ctypes.byref(g), _p(base), base.shape[1], _p(q), nq, _p(tk),
                                                        _p(qu), k_stride, metric, _p(thr), thr.size, _p(out), _p(st),
                                                        threads)
        if rc == -2:
            raise EarlyStopNotRepresentable("Early-stop threshold is not representable in query distance units")
    else:
        rc = oracle_lib().oracle_batch_query(ctypes.byref(g), _p(base), base.shape[1], _p(q), nq, _p(tk), _p(qu),
                                             k_stride, metric, 1 if l0_only else 0, _p(out), _p(st), threads)
    if rc != 0:
        raise ValueError("oracle_batch_query rejected its arguments")
    return (out, st) if stats else out


def bruteforce(base: np.ndarray, queries: np.ndarray, k: int, metric: int = 0, threads: int = None):
    """Exact top-k by (distance, vid): (ids (nq,k) uint32, dists (nq,k) float32)."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    ids = np.empty((q.shape[0], k), dtype=np.uint32)
    d = np.empty((q.shape[0], k), dtype=np.float32)
    rc = oracle_lib().oracle_bruteforce(_p(base), base.shape[0], base.shape[1], _p(q), q.shape[0], k, metric,
                                        _p(ids), _p(d), threads or os.cpu_count() or 1)
    if rc != 0:
        raise ValueError("oracle_bruteforce rejected its arguments")
    return ids, d


def centroid_entry(base: np.ndarray, metric: int, bucket=None) -> int:
    """C restatement of the compactor's centroid entry point."""
    base = np.ascontiguousarray(base, dtype=np.float32)
    b = None if bucket is None else np.ascontiguousarray(bucket, dtype=np.uint32)
    n = base.shape[0] if b is None else b.size
    return int(oracle_lib().oracle_centroid_entry(_p(base), base.shape[1], _p(b), n, metric))


class RefRouter:
    """The reference's hierarchical_graph_router_t over an HGRA snapshot."""

    def __init__(self, hgra_path: str, base: np.ndarray):
        self.base = np.ascontiguousarray(base, dtype=np.float32)
        L = ref_lib()
        self._h = L.artea_ref_open(os.fsencode(hgra_path), _p(self.base), self.base.shape[0], self.base.shape[1])
        if not self._h:
            raise RuntimeError(L.artea_ref_last_error().decode())

    def batch_query(self, queries: np.ndarray, topk: int, queue: int, metric: int = 0, l0_only: bool = False,
                    threads: int = 0, count_distances: bool = False):
        """Returns (words (nq, topk) uint64, seconds[, dist_calls (nq,) uint64])."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        out = np.empty((q.shape[0], topk), dtype=np.uint64)
        secs = c_double()
        calls = np.zeros(q.shape[0], dtype=np.uint64) if count_distances else None
        rc = ref_lib().artea_ref_batch_query(self._h, _p(q), q.shape[0], topk, queue, metric, 1 if l0_only else 0,
                                             threads, _p(out), ctypes.byref(secs), _p(calls))
        if rc != 0:
            raise RuntimeError(ref_lib().artea_ref_last_error().decode())
        return (out, secs.value, calls) if count_distances else (out, secs.value)

    def batch_query_early_stop(self, queries: np.ndarray, topk: int, queue: int, thresholds, metric: int = 0,
                               count_distances: bool = False):
        """batch_query<false, true> with per-level configuration thresholds.
        Returns words (nq, topk) [, dist_calls (nq,)]."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        thr = np.ascontiguousarray(thresholds, dtype=np.float32)
        out = np.empty((q.shape[0], topk), dtype=np.uint64)
        calls = np.zeros(q.shape[0], dtype=np.uint64) if count_distances else None
        rc = ref_lib().artea_ref_batch_query_early_stop(self._h, _p(q), q.shape[0], topk, queue, metric, _p(thr),
                                                        thr.size, _p(out), _p(calls))
        if rc == -2:
            raise EarlyStopNotRepresentable(ref_lib().artea_ref_last_error().decode())
        if rc != 0:
            raise RuntimeError(ref_lib().artea_ref_last_error().decode())
        return (out, calls) if count_distances else out

    def bruteforce(self, queries: np.ndarray, topk: int, metric: int = 0, subset=None) -> np.ndarray:
        """The reference's bruteforce_router_t batch_query (with subset: the subset
        overload): (nq, topk) words, CandidateEntry() padding."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        sub = None if subset is None else np.ascontiguousarray(subset, dtype=np.uint32)
        out = np.empty((q.shape[0], topk), dtype=np.uint64)
        rc = ref_lib().artea_ref_bruteforce(self._h, _p(q), q.shape[0], topk, metric, _p(sub),
                                            0 if sub is None else sub.size, _p(out))
        if rc != 0:
            raise RuntimeError(ref_lib().artea_ref_last_error().decode())
        return out

    def close(self):
        if self._h:
            ref_lib().artea_ref_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def recall_at_k(pred_words: np.ndarray, gt_ids: np.ndarray, k) -> float:
    """recall@k as utils/recall_estimator.hpp:150-230 computes it: per query the
    size of set(pred[:k]) intersected with set(gt[:k]); summed over queries and
    divided by the sum of k. k may be per query."""
    pred = (np.asarray(pred_words, dtype=np.uint64) & np.uint64(0x7FFFFFFF)).astype(np.int64)
    nq = pred.shape[0]
    ks = np.broadcast_to(np.asarray(k), (nq,))
    hits = 0
    for i in range(nq):
        kk = int(ks[i])
        p = set(int(x) for x in pred[i, :kk] if x != 0x7FFFFFFF)
        g = set(int(x) for x in gt_ids[i, :kk])
        hits += len(p & g)
    return hits / float(ks.sum())
