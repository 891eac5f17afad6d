"""Python mirror of the reference router surface, backed by the B200 kernels.

``HierarchicalGraphRouter`` follows hierarchical_graph_router_t<Metric, Dim>
(router/hierarchical_graph_router.hpp:66-430): constructed from the base
vectors, a metric, topk and the candidate queue size (raising like the
reference's ARTEA_ERROR when queue < topk), ``initialize()``, then
``batch_query(query_vecs, graph)`` returning the knn_results_t layout: nq*k
8-byte CandidateEntry words, row-major, invalid-filled. The graph is uploaded
on first use and kept device resident, keyed by the graph object.

There is no CPU path: every call goes through libartea_gpu.so.
"""

from __future__ import annotations

import ctypes
import weakref
from typing import Optional

import numpy as np

from . import _native as nat
from .graph import INVALID_LEVEL, CompactHierarchicalGraph

METRICS = {
    "euclidean_sqr": nat.METRIC_EUCLIDEAN_SQR,
    "l2sq": nat.METRIC_EUCLIDEAN_SQR,
    "euclidean": nat.METRIC_EUCLIDEAN,
    "cosine": nat.METRIC_COSINE,
    "dot": nat.METRIC_DOT,
}
MODES = {"exact": nat.MODE_EXACT, "fast": nat.MODE_FAST}
SCHEDULES = {"auto": nat.SCHEDULE_AUTO, "plain": nat.SCHEDULE_PLAIN, "persistent": nat.SCHEDULE_PERSISTENT}

INVALID_WORD = np.uint64((0x7F7FFFFF << 32) | 0x7FFFFFFF)


def entry_vids(words: np.ndarray) -> np.ndarray:
    """CandidateEntry::get_vid (candidate_entry.hpp:115-118)."""
    return (np.asarray(words, dtype=np.uint64) & np.uint64(0x7FFFFFFF)).astype(np.uint32)


def entry_dists(words: np.ndarray) -> np.ndarray:
    """CandidateEntry::get_distance."""
    return (np.asarray(words, dtype=np.uint64) >> np.uint64(32)).astype(np.uint32).view(np.float32)


def entry_is_invalid(words: np.ndarray) -> np.ndarray:
    """CandidateEntry::is_invalid (candidate_entry.hpp:122-125)."""
    return entry_vids(words) == 0x7FFFFFFF


def metric_code(metric) -> int:
    if isinstance(metric, str):
        return METRICS[metric.lower()]
    return int(metric)


def _result_buffer(nq: int, k_stride: int) -> np.ndarray:
    """(nq, k_stride) uint64 result rows in page-locked memory (torch's caching
    host allocator), which the kernel writes in place: the results reach the
    host while the search runs instead of in a copy after it."""
    if nq * k_stride == 0:
        return np.empty((nq, k_stride), dtype=np.uint64)
    import torch
    t = torch.empty(nq * k_stride, dtype=torch.int64, pin_memory=True)
    return t.numpy().view(np.uint64).reshape(nq, k_stride)


class DeviceIndex:
    """A compact graph plus its FP32 vectors, uploaded once to one GPU."""

    def __init__(self, graph: CompactHierarchicalGraph, base_vecs: np.ndarray, device: int = 0):
        base = np.ascontiguousarray(base_vecs, dtype=np.float32)
        if base.ndim != 2:
            raise ValueError("base_vecs must be a 2-D array")
        self.num_vectors, self.dim = base.shape
        self.device = device
        d = graph.desc()
        h = ctypes.c_void_p()
        nat.check(nat.lib().artea_gpu_index_create(ctypes.byref(d), nat.ptr(base), self.num_vectors, self.dim,
                                                   device, ctypes.byref(h)))
        self._h = h

    @classmethod
    def from_hgra(cls, path: str, base_vecs: np.ndarray, device: int = 0) -> "DeviceIndex":
        self = cls.__new__(cls)
        base = np.ascontiguousarray(base_vecs, dtype=np.float32)
        self.num_vectors, self.dim = base.shape
        self.device = device
        h = ctypes.c_void_p()
        import os
        nat.check(nat.lib().artea_gpu_index_create_from_hgra(os.fsencode(path), nat.ptr(base), self.num_vectors,
                                                             self.dim, device, ctypes.byref(h)))
        self._h = h
        return self

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise RuntimeError("index is closed")
        return self._h

    def download_graph(self, num_vertices: int, num_offsets: int, num_neighbor_ids: int):
        """The device graph as (vertex_info (n, 2) uint32, offsets (all groups
        concatenated) uint64, neighbor_ids uint32), sized as artea_gpu_hgra_probe
        reports them (artea_gpu_index_download)."""
        vinfo = np.empty((num_vertices, 2), dtype=np.uint32)
        offs = np.empty(num_offsets, dtype=np.uint64)
        nbrs = np.empty(max(num_neighbor_ids, 1), dtype=np.uint32)
        nat.check(nat.lib().artea_gpu_index_download(self.handle, nat.ptr(vinfo), nat.ptr(offs), nat.ptr(nbrs)))
        return vinfo, offs, nbrs[:num_neighbor_ids]

    def nbytes(self) -> int:
        b = ctypes.c_uint64()
        nat.check(nat.lib().artea_gpu_index_bytes(self.handle, ctypes.byref(b)))
        return int(b.value)

    def bruteforce(self, queries: np.ndarray, topk: int, metric, subset: Optional[np.ndarray] = None) -> np.ndarray:
        """Exact brute-force top-k over this index's vectors (artea_gpu_bruteforce):
        (nq, topk) CandidateEntry words, ascending, CandidateEntry() padding."""
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, self.dim)
        sub = None if subset is None else np.ascontiguousarray(subset, dtype=np.uint32)
        out = np.empty((q.shape[0], topk), dtype=np.uint64)
        nat.check(nat.lib().artea_gpu_bruteforce(self.handle, metric_code(metric), nat.ptr(q), q.shape[0], topk,
                                                 nat.ptr(sub), 0 if sub is None else sub.size, nat.ptr(out)))
        return out

    def subsystem_probe(self, d_queries, nq: int, topk: int, queue: int, metric, mode: str = "exact",
                        visited_hash_bits: int = 9) -> dict:
        """The query path's subsystems run one at a time on a real search's
        accesses (artea_gpu_subsystem_probe): per-probe milliseconds, work
        recorded and the replays' mismatch counts (all 0 when faithful)."""
        r = nat.ProbeResult()
        nat.check(nat.lib().artea_gpu_subsystem_probe(self.handle, metric_code(metric), MODES[mode], topk, queue,
                                                      nat.ptr(d_queries), nq, visited_hash_bits, ctypes.byref(r)))
        return {name: getattr(r, name) for name, _ in nat.ProbeResult._fields_}

    def centroid_entry(self, metric, bucket: Optional[np.ndarray] = None) -> int:
        """The compactor's entry point: the bucket vid nearest to the bucket's
        centroid (artea_gpu_centroid_entry); 0xFFFFFFFF for an empty bucket."""
        b = None if bucket is None else np.ascontiguousarray(bucket, dtype=np.uint32)
        out = ctypes.c_uint32()
        nat.check(nat.lib().artea_gpu_centroid_entry(self.handle, metric_code(metric), nat.ptr(b),
                                                     0 if b is None else b.size, ctypes.byref(out)))
        return int(out.value)

    def bruteforce_device(self, d_queries, nq: int, topk: int, metric, d_out, d_subset=None, n_subset: int = 0,
                          stream: int = 0) -> None:
        """artea_gpu_bruteforce_device on device buffers (torch tensors or addresses)."""
        nat.check(nat.lib().artea_gpu_bruteforce_device(self.handle, metric_code(metric), nat.ptr(d_queries), nq,
                                                        topk, nat.ptr(d_subset), n_subset, nat.ptr(d_out),
                                                        ctypes.c_void_p(stream or None)))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            nat.lib().artea_gpu_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vectors_only_graph() -> CompactHierarchicalGraph:
    """An empty compact graph: a DeviceIndex over it holds vectors only."""
    return CompactHierarchicalGraph(0, 0, 4, 4, 0xFFFFFFFF, np.zeros((0, 2), np.uint32), [np.zeros(1, np.uint64)],
                                    np.zeros(0, np.uint32))


class BruteforceRouter:
    """Drop-in for bruteforce_router_t<Metric, Dim> (router/bruteforce_router.hpp):
    exact k-NN over base_vecs on the GPU, distances bit-identical to the
    reference's; equal distances come in vid order."""

    def __init__(self, base_vecs: np.ndarray, metric, topk: int, device: int = 0):
        self.base_vecs = base_vecs
        self.metric = metric_code(metric)
        self.topk = int(topk)
        self.device = device
        self._index = None

    def initialize(self) -> None:
        """bruteforce_router.hpp:63-65 (nothing to prepare); the vectors are uploaded on first use."""
        nat.lib()

    def _ix(self) -> DeviceIndex:
        if self._index is None:
            self._index = DeviceIndex(vectors_only_graph(), self.base_vecs, self.device)
        return self._index

    def query(self, query_vec: np.ndarray, subset: Optional[np.ndarray] = None) -> np.ndarray:
        """query (:74-96) / query with subset (:100-125): min(topk, candidates) words."""
        n = self._ix().num_vectors if subset is None else len(subset)
        words = self._ix().bruteforce(np.asarray(query_vec, dtype=np.float32).reshape(1, -1), self.topk,
                                      self.metric, subset)[0]
        return words[: min(self.topk, n)]

    def batch_query(self, query_vecs: np.ndarray, subset: Optional[np.ndarray] = None) -> np.ndarray:
        """batch_query (:130-160, subset :164-190): (nq * topk,) words, CandidateEntry() padding."""
        return self._ix().bruteforce(query_vecs, self.topk, self.metric, subset).reshape(-1)

    def close(self) -> None:
        if self._index is not None:
            self._index.close()
            self._index = None


class GpuRouter:
    """A router handle bound to one DeviceIndex (artea_gpu_router_create)."""

    def __init__(self, index: DeviceIndex, metric, topk: int, candidate_queue_size: int, mode: str = "exact",
                 schedule: str = "auto", warps_per_cta: int = 0, ctas_per_sm: int = 0, max_batch: int = 0,
                 max_queue: int = 0, visited_hash_bits: int = 0, register_budget: int = 0,
                 use_graphs: bool = False, stage_rows: int = 0, pipeline: int = 0, prefetch_rows: int = 0,
                 order_queries: int = 0, warps_per_query: int = 0, queue_slack: int = 0):
        opts = nat.RouterOpts()
        opts.metric = metric_code(metric)
        opts.mode = MODES[mode] if isinstance(mode, str) else int(mode)
        opts.schedule = SCHEDULES[schedule] if isinstance(schedule, str) else int(schedule)
        opts.warps_per_cta = warps_per_cta
        opts.ctas_per_sm = ctas_per_sm
        opts.max_batch = max_batch
        opts.max_queue = max_queue
        opts.visited_hash_bits = visited_hash_bits
        opts.register_budget = register_budget
        opts.stage_rows = stage_rows
        opts.pipeline = pipeline
        opts.prefetch_rows = prefetch_rows
        opts.order_queries = order_queries
        opts.warps_per_query = warps_per_query
        opts.queue_slack = queue_slack
        opts.use_graphs = 1 if use_graphs else 0
        h = ctypes.c_void_p()
        nat.check(nat.lib().artea_gpu_router_create(index.handle, topk, candidate_queue_size, ctypes.byref(opts),
                                                    ctypes.byref(h)))
        self.index = index
        self.topk = topk
        self.queue = candidate_queue_size
        self._h = h

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def batch_query(self, queries: np.ndarray, topk: Optional[np.ndarray] = None, queue: Optional[np.ndarray] = None,
                    k_stride: Optional[int] = None, stats: bool = False, l0_only: bool = False):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim != 2 or q.shape[1] != self.index.dim:
            raise ValueError(f"queries must be (nq, {self.index.dim})")
        nq = q.shape[0]
        tk = None if topk is None else np.ascontiguousarray(topk, dtype=np.uint32)
        qu = None if queue is None else np.ascontiguousarray(queue, dtype=np.uint32)
        if k_stride is None:
            k_stride = int(tk.max()) if tk is not None and tk.size else self.topk
        out = _result_buffer(nq, max(k_stride, 0))
        st = (nat.QueryStats * max(nq, 1))() if stats else None
        L = nat.lib()
        if l0_only:
            if tk is not None or qu is not None:
                raise ValueError("l0_only takes the router's topk and queue")
            rc = L.artea_gpu_batch_query_l0_only(self._h, nat.ptr(q), nq, k_stride, nat.ptr(out),
                                                 ctypes.cast(st, ctypes.c_void_p) if st is not None else None)
        else:
            rc = L.artea_gpu_batch_query(self._h, nat.ptr(q), nq, nat.ptr(tk), nat.ptr(qu), k_stride,
                                         nat.ptr(out), ctypes.cast(st, ctypes.c_void_p) if st is not None else None)
        nat.check(rc)
        if stats:
            arr = np.ctypeslib.as_array(st)[:nq]
            return out, np.array(arr.tolist(), dtype=np.uint32).reshape(nq, 8)
        return out

    def batch_query_device(self, d_queries, nq: int, k_stride: int, d_out, d_topk=None, d_queue=None, d_stats=None,
                           stream: int = 0) -> None:
        """Enqueue on device buffers (torch tensors or raw addresses); no sync."""
        nat.check(nat.lib().artea_gpu_batch_query_device(self._h, nat.ptr(d_queries), nq, nat.ptr(d_topk),
                                                         nat.ptr(d_queue), k_stride, nat.ptr(d_out),
                                                         nat.ptr(d_stats), ctypes.c_void_p(stream or None)))

    def sync(self) -> None:
        nat.check(nat.lib().artea_gpu_router_sync(self._h))

    def set_early_stop(self, level_thresholds) -> None:
        """enable_early_stop=true for later launches: level_thresholds[h] is the
        configuration's early_stop_threshold(h, pruning) (index 0 unused); None
        switches it off. OverflowError when a threshold is not representable in
        query units (hierarchical_graph_router.hpp:398-404)."""
        if level_thresholds is None:
            nat.check(nat.lib().artea_gpu_router_set_early_stop(self._h, None, 0))
            return
        thr = np.ascontiguousarray(level_thresholds, dtype=np.float32)
        rc = nat.lib().artea_gpu_router_set_early_stop(self._h, nat.ptr(thr), thr.size)
        if rc == nat.EINVAL:
            msg = nat.lib().artea_gpu_last_error().decode(errors="replace")
            if "not representable" in msg:
                raise OverflowError(msg)
        nat.check(rc)

    def set_phase_buffer(self, d_buf) -> None:
        """Record per-query phase cycles into d_buf (device, nq x 8 int64) or stop (None)."""
        nat.check(nat.lib().artea_gpu_router_set_phase_buffer(self._h, nat.ptr(d_buf)))

    def tuning(self) -> dict:
        """Launch parameters of the last launch (the autotuner's pick)."""
        w, b, g, st = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        nat.check(nat.lib().artea_gpu_router_tuning(self._h, ctypes.byref(w), ctypes.byref(b), ctypes.byref(g),
                                                    ctypes.byref(st)))
        p, pf, o, q, sl = (ctypes.c_uint32() for _ in range(5))
        nat.check(nat.lib().artea_gpu_router_tuning_ext(self._h, ctypes.byref(p), ctypes.byref(pf), ctypes.byref(o),
                                                        ctypes.byref(q), ctypes.byref(sl)))
        return {"warps_per_cta": w.value, "visited_hash_bits": b.value, "register_budget": g.value,
                "stage_rows": st.value, "pipeline": p.value, "prefetch_rows": pf.value, "ordered": o.value,
                "warps_per_query": q.value, "queue_slack": sl.value}

    def last_reruns(self) -> int:
        """Queries of the last compact-queue launch rerun at full capacity (waits)."""
        n = ctypes.c_uint32()
        nat.check(nat.lib().artea_gpu_router_last_reruns(self._h, ctypes.byref(n)))
        return int(n.value)

    def launches(self) -> int:
        n = ctypes.c_uint64()
        nat.check(nat.lib().artea_gpu_router_launches(self._h, ctypes.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            nat.lib().artea_gpu_router_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HierarchicalGraphRouter:
    """Drop-in for hierarchical_graph_router_t<Metric, Dim>.

    ``base_vecs`` is held by reference, as the reference router holds a const
    reference (router/vector_router.hpp:46, 63-69). ``batch_query`` takes the
    graph per call; the first call with a graph uploads it (with the vectors)
    and later calls reuse the device copy.
    """

    def __init__(self, base_vecs: np.ndarray, metric, topk: int, candidate_queue_size: int = 16,
                 mode: str = "exact", schedule: str = "auto", device: int = 0, **router_opts):
        if candidate_queue_size < topk:
            # hierarchical_graph_router.hpp:104-108 (ARTEA_ERROR throws std::runtime_error)
            raise RuntimeError(f"candidate_queue_size ({candidate_queue_size}) must be >= topk ({topk})")
        self.base_vecs = base_vecs
        self.metric = metric_code(metric)
        self.topk = int(topk)
        self.candidate_queue_size = int(candidate_queue_size)
        self.mode = mode
        self.schedule = schedule
        self.device = device
        self.router_opts = router_opts
        self._cache = {}

    def initialize(self) -> None:
        """hierarchical_graph_router.hpp:114-117; device state is created lazily per graph."""
        nat.lib()

    def _router_for(self, graph: CompactHierarchicalGraph) -> GpuRouter:
        key = id(graph)
        hit = self._cache.get(key)
        if hit is not None and hit[0]() is graph:
            return hit[1]
        index = DeviceIndex(graph, self.base_vecs, self.device)
        router = GpuRouter(index, self.metric, self.topk, self.candidate_queue_size, mode=self.mode,
                           schedule=self.schedule, **self.router_opts)
        self._cache[key] = (weakref.ref(graph), router)
        return router

    def _early_stop(self, router: GpuRouter, graph: CompactHierarchicalGraph, enable_early_stop: bool,
                    rgraph_config, pruning_config) -> None:
        """_early_stop_thresholds (hierarchical_graph_router.hpp:388-408): one
        rgraph_config.early_stop_threshold(h, pruning_config) per upper level,
        converted and validated by the native router."""
        if not enable_early_stop:
            router.set_early_stop(None)
            return
        top = graph.top_occupied_level_id()
        if graph.num_vertices == 0 or top == INVALID_LEVEL or top == 0:
            router.set_early_stop(None)
            return
        if rgraph_config is None or pruning_config is None:
            raise TypeError("early stopping on a bare graph requires explicit rgraph and pruning configs")
        thr = [0.0] + [float(rgraph_config.early_stop_threshold(h, pruning_config)) for h in range(1, top + 1)]
        router.set_early_stop(thr)

    def batch_query(self, query_vecs: np.ndarray, graph: CompactHierarchicalGraph, rgraph_config=None,
                    pruning_config=None, enable_early_stop: bool = False) -> np.ndarray:
        """knn_results_t: (nq * topk,) uint64 CandidateEntry words. With
        enable_early_stop, the config overload (hierarchical_graph_router.hpp:308-319)."""
        r = self._router_for(graph)
        self._early_stop(r, graph, enable_early_stop, rgraph_config, pruning_config)
        out = r.batch_query(query_vecs)
        return out.reshape(-1)

    def query(self, query_vec: np.ndarray, graph: CompactHierarchicalGraph, rgraph_config=None,
              pruning_config=None, enable_early_stop: bool = False) -> np.ndarray:
        """query(): at most topk entries (the invalid tail is dropped)."""
        r = self._router_for(graph)
        self._early_stop(r, graph, enable_early_stop, rgraph_config, pruning_config)
        words = r.batch_query(np.asarray(query_vec, dtype=np.float32).reshape(1, -1))[0]
        return words[~entry_is_invalid(words)]

    def batch_query_l0_only(self, query_vecs: np.ndarray, graph: CompactHierarchicalGraph) -> np.ndarray:
        out = self._router_for(graph).batch_query(query_vecs, l0_only=True)
        return out.reshape(-1)

    def close(self) -> None:
        for _, (_, r) in list(self._cache.items()):
            r.close()
            r.index.close()
        self._cache.clear()
