"""Serving loop: continuous batching over the device-resident index.

``Server`` wraps artea_gpu_server_* (include/artea_gpu.h): requests of any
size are admitted while the device ring has room, folded into the running
persistent kernel and polled for completion. ``run_poisson`` drives a server
with Poisson request arrivals and reports latency percentiles and throughput;
``run_per_batch`` is the comparison point that launches one batch_query per
request, one after another.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _native as nat
from .router import DeviceIndex, GpuRouter, metric_code, MODES


class Server:
    def __init__(self, index: DeviceIndex, metric, max_topk: int, max_queue: int, ring_slots: int = 16384,
                 mode: str = "exact", warps_per_cta: int = 0, idle_polls: int = 0, heartbeat_ms: int = 0):
        o = nat.ServerOpts()
        o.metric = metric_code(metric)
        o.mode = MODES[mode]
        o.max_topk = max_topk
        o.max_queue = max_queue
        o.ring_slots = ring_slots
        o.warps_per_cta = warps_per_cta
        o.idle_polls = idle_polls
        o.heartbeat_ms = heartbeat_ms
        h = ctypes.c_void_p()
        nat.check(nat.lib().artea_gpu_server_create(index.handle, ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.index = index
        self.max_topk = max_topk

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def submit(self, queries: np.ndarray, topk: Optional[np.ndarray] = None,
               queue: Optional[np.ndarray] = None) -> Optional[int]:
        """Ticket of the admitted request, or None when the ring is full."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        tk = None if topk is None else np.ascontiguousarray(topk, dtype=np.uint32)
        qu = None if queue is None else np.ascontiguousarray(queue, dtype=np.uint32)
        t = ctypes.c_uint64()
        rc = nat.lib().artea_gpu_server_submit(self._h, nat.ptr(q), q.shape[0], nat.ptr(tk), nat.ptr(qu),
                                               ctypes.byref(t))
        if rc == nat.EBUSY:
            return None
        nat.check(rc)
        return int(t.value)

    def poll(self, ticket: int, n: int, k_stride: Optional[int] = None) -> Optional[np.ndarray]:
        """(n, k_stride) result words once the request finished, else None."""
        k = self.max_topk if k_stride is None else k_stride
        out = np.empty((n, k), dtype=np.uint64)
        done = ctypes.c_int()
        nat.check(nat.lib().artea_gpu_server_poll(self._h, ticket, n, k, nat.ptr(out), ctypes.byref(done)))
        return out if done.value else None

    def wait(self, ticket: int, n: int, k_stride: Optional[int] = None, timeout_s: float = 60.0) -> np.ndarray:
        t0 = time.perf_counter()
        while True:
            r = self.poll(ticket, n, k_stride)
            if r is not None:
                return r
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError(f"request {ticket} not finished after {timeout_s} s")

    def pause_heartbeat(self) -> None:
        """Stop the server's heartbeat, as a host that stopped answering would
        (failure injection: the kernel ends heartbeat_ms later)."""
        nat.check(nat.lib().artea_gpu_server_pause_heartbeat(self._h))

    def stats(self) -> dict:
        p, c, l = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        nat.check(nat.lib().artea_gpu_server_stats(self._h, ctypes.byref(p), ctypes.byref(c), ctypes.byref(l)))
        return {"published": p.value, "consumed": c.value, "kernel_launches": l.value}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            nat.lib().artea_gpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Request:
    arrival: float
    lo: int
    n: int
    topk: np.ndarray
    queue: np.ndarray
    ticket: Optional[int] = None
    finished: Optional[float] = None
    result: Optional[np.ndarray] = field(default=None, repr=False)


def make_requests(nq_total: int, rate_qps: float, seed: int, topk_choices=(10, 100), queue_choices=(100, 200, 400),
                  max_size: int = 256) -> List[Request]:
    """Poisson arrivals at rate_qps queries/s; sizes log-uniform in [1, max_size];
    per-request topk and queue drawn from the choices (queue >= topk)."""
    rng = np.random.default_rng(seed)
    reqs, t, lo = [], 0.0, 0
    while lo < nq_total:
        n = int(min(nq_total - lo, max(1, round(np.exp(rng.uniform(0, np.log(max_size)))))))
        t += rng.exponential(n / rate_qps)
        k = int(rng.choice(topk_choices))
        L = max(int(rng.choice(queue_choices)), k)
        reqs.append(Request(t, lo, n, np.full(n, k, np.uint32), np.full(n, L, np.uint32)))
        lo += n
    return reqs


def latency_percentile(lat, p: float) -> float:
    """The reference profiler's pick (router/profiler/hg_router_profiler.hpp:429-444):
    the sorted sample at index floor(n * p), clamped to the last one; no
    interpolation."""
    s = np.sort(np.asarray(lat, dtype=np.float64))
    if s.size == 0:
        return float("nan")
    return float(s[min(int(s.size * p), s.size - 1)])


def _summarise(reqs: List[Request], wall: float) -> dict:
    lat = np.array([(r.finished - r.arrival) * 1e3 for r in reqs])
    nq = sum(r.n for r in reqs)
    return {"requests": len(reqs), "queries": nq, "qps": nq / wall, "wall_s": wall,
            "p50_ms": latency_percentile(lat, 0.50), "p90_ms": latency_percentile(lat, 0.90),
            "p95_ms": latency_percentile(lat, 0.95), "p99_ms": latency_percentile(lat, 0.99),
            "mean_ms": float(lat.mean())}


def run_poisson(server: Server, queries: np.ndarray, reqs: List[Request], k_stride: int,
                timeout_s: float = 300.0) -> dict:
    """Submit each request at its arrival time (or as soon as the ring has
    room), poll outstanding ones, time arrival -> observed completion."""
    pending = list(reqs)
    outstanding: List[Request] = []
    t0 = time.perf_counter()
    while pending or outstanding:
        now = time.perf_counter() - t0
        if now > timeout_s:
            raise TimeoutError("serving run did not finish")
        while pending and pending[0].arrival <= now:
            r = pending[0]
            tk = server.submit(queries[r.lo:r.lo + r.n], r.topk, r.queue)
            if tk is None:
                break
            r.ticket = tk
            outstanding.append(pending.pop(0))
        still = []
        for r in outstanding:
            res = server.poll(r.ticket, r.n, k_stride)
            if res is None:
                still.append(r)
            else:
                r.finished = time.perf_counter() - t0
                r.result = res
        outstanding = still
    return _summarise(reqs, time.perf_counter() - t0)


def run_per_batch(router: GpuRouter, queries: np.ndarray, reqs: List[Request], k_stride: int) -> dict:
    """Comparison point: one batch_query launch per request, in arrival order."""
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if now < r.arrival:
            time.sleep(r.arrival - now)
        r.result = router.batch_query(queries[r.lo:r.lo + r.n], topk=r.topk, queue=r.queue, k_stride=k_stride)
        r.finished = time.perf_counter() - t0
    return _summarise(reqs, time.perf_counter() - t0)
