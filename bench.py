#!/usr/bin/env python3
"""Benchmark of the B200 hierarchical-graph router (ARTEA batch_query).

Metric: QPS at recall@100 >= 0.95. The default workload is the 1M x 128
Euclidean SIFT-like index (seeded synthetic stand-in, 10,000 queries, topk
100): the queue size is swept over {100, 200, 400, 800} and the smallest size
whose recall@100 reaches 0.95 is timed. One step = one batch_query of all
10,000 queries.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device time (CUDA events around each launch on its stream, inputs
already in HBM, L2 flushed between steps and excluded); `e2e` is the same
metric through the public C-ABI with host buffers inside the timed region: the
queries sit in page-locked host memory and the router returns its results in
page-locked memory, so the kernel reads the queries and writes the result rows
across the bus while it searches (pageable buffers would be staged by copies). Multi-GPU runs are replicas (weak scaling):
every rank holds the whole index and answers its own batch.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from artea_b200 import datasets as ds  # noqa: E402
from artea_b200 import workload as wl  # noqa: E402

METRIC_NAME = "QPS @ recall@100>=0.95"
DEFAULT_QUEUES = (100, 200, 400, 800)


def log(msg: str) -> None:
    if int(os.environ.get("RANK", "0")) == 0:
        print(f"[bench] {msg}", file=sys.stderr, flush=True)


def host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(f in flags for f in ("avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd"))
    except OSError:
        return False


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def metric_code(name: str) -> int:
    return {"euclidean": 0, "cosine": 2, "dot": 3}[name]


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0: float, t1: float) -> None:
        """Keep the samples taken between t0 and t1 (time.time())."""
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        lines = self.lines
        if self.window is not None:
            inside = [l for l in lines if self.window[0] <= l[0] <= self.window[1] + 0.15]
            lines = inside or lines
        for _, line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm.append(float(parts[2]))
                mx = max(mx, float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Ground truth: the exact brute-force top-k of the search metric (the
# reference's bruteforce_router_t semantics, distances bit-identical), computed
# by artea_gpu_bruteforce on the uploaded index; equal distances in vid order.
# ---------------------------------------------------------------------------
def ground_truth(index, base: np.ndarray, queries: np.ndarray, k: int, metric: str, cache_dir: str) -> np.ndarray:
    path = os.path.join(cache_dir, f"gtbf-{metric}-{k}-{ds.fingerprint(base)}-{ds.fingerprint(queries)}.npy")
    if os.path.exists(path):
        return np.load(path)
    out = np.empty((queries.shape[0], k), dtype=np.uint32)
    for lo in range(0, queries.shape[0], 2048):
        words = index.bruteforce(queries[lo:lo + 2048], k, metric_code(metric))
        out[lo:lo + 2048] = (words & np.uint64(0x7FFFFFFF)).astype(np.uint32)
    os.makedirs(cache_dir, exist_ok=True)
    np.save(path, out)
    return out


def recall(words: np.ndarray, gt: np.ndarray, k) -> float:
    pred = (words & np.uint64(0x7FFFFFFF)).astype(np.int64)
    ks = np.broadcast_to(np.asarray(k), (pred.shape[0],))
    hits = 0
    for i in range(pred.shape[0]):
        kk = int(ks[i])
        hits += len(set(pred[i, :kk].tolist()) & set(gt[i, :kk].tolist()))
    return hits / float(ks.sum())


def algorithmic_bytes(stats: np.ndarray, dim: int, k) -> np.ndarray:
    """Bytes one query must move: its query row, one vector row per distance
    evaluation, per row read the vertex record (8 B) and two CSR offsets
    (16 B) plus 4 B per neighbour id, and its k result entries (8 B each)."""
    st = stats.astype(np.float64)
    rows = st[:, 1] + st[:, 3]
    ids = st[:, 2] + st[:, 4]
    return 4.0 * dim + st[:, 0] * 4.0 * dim + rows * 24.0 + ids * 4.0 + 8.0 * np.asarray(k, dtype=np.float64)


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic(workload: str, queue=None):
    """dram read+write bytes per launch from the committed ncu summary of this
    workload: the line for this queue size (traffic_bytes_per_launch_L<queue>:)
    if there is one, else the workload's default line (traffic_bytes_per_launch:)."""
    p = os.path.join(ROOT, "profiles", f"search_kernel_{workload}.md")
    if not os.path.exists(p):
        return None
    keys = ([f"traffic_bytes_per_launch_L{queue}:"] if queue is not None else []) + ["traffic_bytes_per_launch:"]
    lines = [line.strip() for line in open(p)]
    for key in keys:
        for line in lines:
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own batch_query on this host's cores.
# ---------------------------------------------------------------------------
def cpu_baseline(hgra: str, base: np.ndarray, queries: np.ndarray, topk: int, queue: int, metric: int,
                 sample: int, repeats: int = 1) -> dict:
    from oracle import oracle as orc
    q = queries[:sample]
    threads = os.cpu_count() or 1
    if orc.have_ref() and host_has_avx512():
        r = orc.RefRouter(hgra, base)
        r.batch_query(q[: min(256, len(q))], topk, queue, metric=metric)   # warm-up
        secs = []
        for _ in range(repeats):
            _, s = r.batch_query(q, topk, queue, metric=metric)
            secs.append(s)
        cores = int(orc.ref_lib().artea_ref_max_threads())
        r.close()
        kind = "reference"
    else:
        from artea_b200.graph import CompactHierarchicalGraph
        g = CompactHierarchicalGraph.from_hgra(hgra)
        orc.batch_query(g, base, q[: min(256, len(q))], topk, queue, metric=metric, threads=threads)
        secs = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            orc.batch_query(g, base, q, topk, queue, metric=metric, threads=threads)
            secs.append(time.perf_counter() - t0)
        cores = threads
        kind = "port"
    s = statistics.mean(secs)
    return {"value": len(q) / s, "unit": "queries/s", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{len(q)} queries x {repeats} run(s) of batch_query at queue {queue}, topk {topk}",
            "seconds_per_run": s}


# ---------------------------------------------------------------------------
def reference_queue(args, w, base, queries, hgra, metric: int):
    """The queue the GPU arm's sweep settles on: the first of --queues whose
    recall@k reaches --recall-target, else the largest. EXACT mode returns the
    reference's words, so the reference's own recall at a queue is the GPU
    arm's; it is measured here on the first --reference-select queries
    against the reference's brute force (bruteforce_router_t)."""
    if args.reference_queue:
        return args.reference_queue, "given by --reference-queue"
    from oracle import oracle as orc
    queues = [int(x) for x in args.queues.split(",") if x]
    q = queries[: min(args.reference_select, queries.shape[0])]
    k = w.topk
    use_ref = orc.have_ref() and host_has_avx512()
    if use_ref:
        r = orc.RefRouter(hgra, base)
        gt = (r.bruteforce(q, k, metric) & np.uint64(0x7FFFFFFF)).astype(np.uint32)
    else:
        from artea_b200.graph import CompactHierarchicalGraph
        g = CompactHierarchicalGraph.from_hgra(hgra)
        gt = orc.bruteforce(base, q, k, metric=metric)[0]
    chosen, seen = queues[-1], []
    for L in queues:
        if use_ref:
            words, _ = r.batch_query(q, k, L, metric=metric)
        else:
            words = orc.batch_query(g, base, q, k, L, metric=metric, threads=os.cpu_count() or 1)
        rec = recall(words, gt, k)
        seen.append(f"{L}: {rec:.4f}")
        if rec >= args.recall_target:
            chosen = L
            break
    if use_ref:
        r.close()
    return chosen, (f"first queue with recall@{k} >= {args.recall_target} on {q.shape[0]} queries against "
                    f"brute force ({', '.join(seen)})")


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, base, queries, hgra, report = wl.prepare(args.workload, args.n_base, args.n_query, log=log)
    metric = metric_code(w.metric)
    sample = min(args.reference_sample, queries.shape[0])
    uneven = args.uneven or w.kind == "deep"
    if uneven:
        # The GPU arm's uneven batch: per-query topk and queue, same draws.
        topk, queue = ds.per_query_params(w, queries.shape[0])
        cfg = {"topk": "per query in {10,100}", "queue": "per query in {64,128,256,512}"}
        timed = lambda: cpu_baseline_uneven(hgra, base, queries, topk, queue, metric, sample)
    else:
        queue, why = reference_queue(args, w, base, queries, hgra, metric)
        cfg = {"topk": w.topk, "queue": queue, "queue_selection": why}
        timed = lambda: cpu_baseline(hgra, base, queries, w.topk, queue, metric, sample)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = timed()
        if i >= args.warmup:
            vals.append(info["value"])
    value = statistics.mean(vals)
    line = {"metric": METRIC_NAME, "value": value, "unit": "queries/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sample / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": w.name, "n_base": w.n_base, "n_query": sample,
                                           "dim": w.dim, "metric": w.metric, **cfg},
            "cpu_baseline": {k: info[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model")},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_steps(router, d_q, nq, k_stride, d_out, d_topk, d_queue, stream, steps, warmup, flush):
    """CUDA-event time (ms) of each of `steps` launches after `warmup` untimed ones;
    the L2 flush between steps is outside the events."""
    import torch
    for _ in range(warmup):
        router.batch_query_device(d_q, nq, k_stride, d_out, d_topk=d_topk, d_queue=d_queue, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ev = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        router.batch_query_device(d_q, nq, k_stride, d_out, d_topk=d_topk, d_queue=d_queue, stream=stream.cuda_stream)
        e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def run_uneven(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world):
    """One launch over queries with uneven per-query topk/queue: the persistent
    schedule (autotuned, work stealing, CUDA graphs) against the plain
    one-CTA-per-query schedule; both must return identical words."""
    import torch
    from artea_b200.router import GpuRouter
    nq, dim = queries.shape
    topk, queue = ds.per_query_params(w, nq)
    kmax = int(topk.max())
    gt = ground_truth(index, base, queries, kmax, w.metric, cache_dir)
    d_q = torch.from_numpy(queries).to(device)
    d_tk = torch.from_numpy(topk.view(np.int32)).to(device)
    d_qu = torch.from_numpy(queue.view(np.int32)).to(device)
    d_out = torch.empty((nq, kmax), dtype=torch.int64, device=device)
    d_stats = torch.zeros((nq, 8), dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    res = {}
    for sched in ("persistent", "plain"):
        r = GpuRouter(index, metric, kmax, int(queue.max()), mode=args.mode, schedule=sched, max_batch=nq,
                      use_graphs=not args.no_graphs)
        r.batch_query_device(d_q, nq, kmax, d_out, d_topk=d_tk, d_queue=d_qu, d_stats=d_stats,
                             stream=stream.cuda_stream)
        torch.cuda.synchronize()
        words = d_out.cpu().numpy().view(np.uint64).copy()
        stats = d_stats.cpu().numpy().view(np.uint32).copy()
        l0 = r.launches()
        with ClockSampler(local_gpu(device)) as clocks:
            time.sleep(0.3)
            t0 = time.time()
            ms = time_steps(r, d_q, nq, kmax, d_out, d_tk, d_qu, stream, args.steps, args.warmup, flush)
            clocks.mark(t0, time.time())
            time.sleep(0.2)
        r.sync()
        res[sched] = {"ms": statistics.mean(ms), "qps": nq / (statistics.mean(ms) / 1e3),
                      "recall": recall(words, gt, topk), "tuning": r.tuning(),
                      "launches": r.launches() - l0 - args.warmup, "stats": stats, "words": words,
                      "clocks": clocks.summary(), "router": r}
        log(f"{sched}: {res[sched]['qps']:.0f} q/s, recall {res[sched]['recall']:.5f}, tuning {r.tuning()}")
    assert np.array_equal(res["persistent"]["words"], res["plain"]["words"]), "schedules disagree"
    p = res["persistent"]
    hq = torch.from_numpy(queries).pin_memory().numpy()   # host queries in page-locked memory, as a server holds them
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        p["router"].batch_query(hq, topk=topk, queue=queue, k_stride=kmax)
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    alg = float(algorithmic_bytes(p["stats"], dim, topk).sum())
    peaks = measured_peaks()
    achieved = alg / (p["ms"] / 1e3) / 1e9
    baseline = None
    if not args.no_cpu_baseline:
        baseline = cpu_baseline_uneven(hgra, base, queries, topk, queue, metric, min(args.cpu_sample, nq))
    st = p["stats"].astype(np.float64)
    line = {
        "metric": METRIC_NAME, "value": p["qps"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": p["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "n_base": w.n_base, "n_query": nq, "dim": dim, "metric": w.metric,
                   "topk": "per query in {10,100}", "queue": "per query in {64,128,256,512}",
                   "mode": args.mode, "schedule": "persistent (autotuned, work stealing)",
                   "cuda_graphs": not args.no_graphs, "recall_at_k": round(p["recall"], 5),
                   "tuning": p["tuning"], "graph_levels": report.get("vertices_by_highest_level"),
                   "graph_build_s": report.get("build_s"),
                   "l2": "256 MiB buffer written between timed steps (excluded from timing)"},
        "plain_one_cta_per_query": {"qps": res["plain"]["qps"], "ms_per_step": res["plain"]["ms"],
                                    "recall_at_k": round(res["plain"]["recall"], 5),
                                    "clocks": res["plain"]["clocks"]},
        "speedup_vs_plain": p["qps"] / res["plain"]["qps"],
        "e2e": {"value": nq / statistics.mean(e2e), "unit": "queries/s",
                "h2d_bytes_per_step": int(queries.nbytes + topk.nbytes + queue.nbytes),
                "d2h_bytes_per_step": int(nq * kmax * 8)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": profile_traffic(w.name),
                     "algorithmic_bytes_per_launch": alg, "peak_source": peaks["source"],
                     "kernel": "search_persistent_kernel"},
        "cpu_baseline": baseline, "gpu_launches": int(p["launches"]), "clocks": p["clocks"],
        "per_query": {"dist_evals": float(st[:, 0].mean()), "l0_rows": float(st[:, 3].mean()),
                      "upper_rows": float(st[:, 1].mean())},
    }
    for sched in res:
        res[sched]["router"].close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline_uneven(hgra, base, queries, topk, queue, metric, sample):
    """The reference router takes one (topk, queue) per instance: the sample is
    grouped by (topk, queue) and each group runs as one batch_query."""
    groups = {}
    for i in range(sample):
        groups.setdefault((int(topk[i]), int(queue[i])), []).append(i)
    total, info = 0.0, None
    for (k, L), idx in sorted(groups.items()):
        info = cpu_baseline(hgra, base, queries[idx], k, L, metric, len(idx))
        total += info["seconds_per_run"]
    return {"value": sample / total, "unit": "queries/s", "cores": info["cores"], "kind": info["kind"],
            "cpu_model": info["cpu_model"],
            "sample": f"{sample} queries in {len(groups)} (topk, queue) groups, one batch_query per group"}


def run_serving(args, w, base, queries, report, index, device, metric, cache_dir):
    """Serving loop under Poisson arrivals against one batch_query per request."""
    from artea_b200.router import GpuRouter
    from artea_b200.serving import Server, make_requests, run_per_batch, run_poisson
    nq = min(args.serve_queries, queries.shape[0])
    qs = queries[:nq]
    gt = ground_truth(index, base, queries, 100, w.metric, cache_dir)[:nq]
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    srv = Server(index, metric, max_topk=100, max_queue=400, ring_slots=16384, mode=args.mode)
    # Untimed first request: the kernel launch and module load stay out of the latencies.
    nw = min(256, nq)
    srv.wait(srv.submit(qs[:nw], topk=np.full(nw, 100, np.uint32), queue=np.full(nw, 400, np.uint32)), nw)
    points = []
    for rate in rates:
        reqs = make_requests(nq, rate, seed=int(rate))
        try:
            st = run_poisson(srv, qs, reqs, 100, timeout_s=120.0)
        except TimeoutError:
            # Recorded, not hidden: the rate's requests did not all finish.
            done = sum(r.n for r in reqs if r.finished is not None)
            points.append({"offered_qps": rate, "stalled": True, "queries_finished": done, "queries": nq,
                           "server_stats": srv.stats()})
            log(f"serving at {rate:.0f} q/s: STALLED after {done} of {nq} queries; later rates skipped")
            break
        order = sorted(reqs, key=lambda r: r.lo)
        words = np.vstack([r.result for r in order])
        ks = np.concatenate([r.topk for r in order])
        st["recall_at_k"] = round(recall(words, gt, ks), 5)
        st["offered_qps"] = rate
        points.append(st)
        log(f"serving at {rate:.0f} q/s: {st}")
    sstats = srv.stats()
    srv.close()
    router = GpuRouter(index, metric, 100, 400, mode=args.mode, schedule="plain", max_batch=256, max_queue=400)
    # Untimed first call: buffer allocation and module load stay out of the latencies.
    router.batch_query(qs[:256], topk=np.full(min(256, nq), 100, np.uint32),
                       queue=np.full(min(256, nq), 400, np.uint32), k_stride=100)
    base_pts = []
    for rate in rates:
        reqs = make_requests(nq, rate, seed=int(rate))
        st = run_per_batch(router, qs, reqs, 100)
        st["offered_qps"] = rate
        base_pts.append(st)
        log(f"per-batch launches at {rate:.0f} q/s: {st}")
    router.close()
    line = {"metric": "serving p50/p95/p99 latency (ms) and QPS at offered load", "unit": "ms", "n_gpus": 1,
            "higher_is_better": False, "data": "synthetic", "dtype": "f32",
            "config": {"workload": w.name, "n_base": w.n_base, "dim": w.dim, "metric": w.metric,
                       "queries_per_rate": nq, "request_size": "log-uniform [1,256]",
                       "topk": "{10,100} per request", "queue": "{100,200,400} per request", "mode": args.mode,
                       "ring_slots": 16384, "arrivals": "Poisson"},
            "serving": points, "server_stats": sstats, "per_batch_launch": base_pts}
    print(json.dumps(line), flush=True)


def run_restore(args, w, base, hgra, device):
    """HGRA snapshot -> searchable device index: the streamed device restore
    (artea_gpu_index_create_from_hgra) against the host reader + upload
    (artea_gpu_hgra_read + artea_gpu_index_create) and the reference's
    HierarchicalGraphFileManager::restore on the host cores. The file is in the
    page cache for every timing; vector uploads are timed alone and reported
    apart, since the reference's restore reads no vectors."""
    import torch
    from artea_b200.graph import CompactHierarchicalGraph
    from artea_b200.router import DeviceIndex, vectors_only_graph
    from oracle import oracle as orc
    with open(hgra, "rb") as f:
        while f.read(1 << 26):
            pass
    reps = max(1, min(args.steps, 5))

    def timed(make):
        out = []
        for i in range(1 + reps):
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            ix = make()
            torch.cuda.synchronize(device)
            dt = time.perf_counter() - t0
            ix.close()
            if i:
                out.append(dt)
        return statistics.median(out)

    dev = local_gpu(device)
    t_stream = timed(lambda: DeviceIndex.from_hgra(hgra, base, device=dev))
    t_host = timed(lambda: DeviceIndex(CompactHierarchicalGraph.from_hgra(hgra), base, device=dev))
    t_vec = timed(lambda: DeviceIndex(vectors_only_graph(), base, device=dev))
    # What is timed is checked: the streamed device graph equals the host reader's.
    g = CompactHierarchicalGraph.from_hgra(hgra)
    ix = DeviceIndex.from_hgra(hgra, base, device=dev)
    offs = np.concatenate(g.group_offsets)
    vi, of, nb = ix.download_graph(g.num_vertices, offs.size, g.neighbor_ids.size)
    same = bool(np.array_equal(vi, g.vertex_info) and np.array_equal(of, offs) and np.array_equal(nb, g.neighbor_ids))
    ix.close()
    assert same, "streamed restore differs from the host reader"
    ref_s, ref_kind = None, None
    if orc.have_ref():
        orc.ref_restore_seconds(hgra)
        ref_s = statistics.median([orc.ref_restore_seconds(hgra) for _ in range(reps)])
        ref_kind = "reference"
    size = os.path.getsize(hgra)
    line = {"metric": "HGRA snapshot restore to a searchable device index", "value": t_stream, "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "steps": reps, "warmup": 1, "data": "synthetic", "dtype": "u32",
            "config": {"workload": w.name, "n_base": w.n_base, "dim": w.dim, "snapshot_bytes": size,
                       "graph_levels": g.group_sizes().tolist(), "page_cache": "warm"},
            "streamed_restore_s": t_stream, "host_reader_then_upload_s": t_host, "vectors_only_s": t_vec,
            "graph_part_streamed_s": t_stream - t_vec, "graph_part_host_s": t_host - t_vec,
            "snapshot_gbs_streamed": size / max(t_stream - t_vec, 1e-9) / 1e9,
            "reference_restore_s": ref_s, "reference_kind": ref_kind,
            "reference_threads": int(orc.ref_lib().artea_ref_max_threads()) if ref_s is not None else None,
            "device_graph_equals_host_reader": same}
    print(json.dumps(line), flush=True)


def local_gpu(device) -> int:
    return device.index if getattr(device, "index", None) is not None else 0


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="sift1m", choices=sorted(ds.WORKLOADS))
    ap.add_argument("--n-base", type=int, default=None)
    ap.add_argument("--n-query", type=int, default=None)
    ap.add_argument("--mode", choices=("exact", "fast"), default="exact")
    ap.add_argument("--schedule", choices=("auto", "plain", "persistent"), default="auto")
    ap.add_argument("--queues", default=",".join(str(q) for q in DEFAULT_QUEUES))
    ap.add_argument("--recall-target", type=float, default=0.95)
    ap.add_argument("--cpu-sample", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graphs", action="store_true", help="launch directly instead of replaying CUDA graphs")
    ap.add_argument("--reference-queue", type=int, default=0)
    ap.add_argument("--reference-sample", type=int, default=2000)
    ap.add_argument("--reference-select", type=int, default=200,
                    help="queries on which the reference arm measures recall to pick its queue")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: one warm and one measured launch at --profile-queue with "
                         "--profile-warps warps per CTA; no sweep, ground truth or baseline")
    ap.add_argument("--profile-queue", type=int, default=200)
    ap.add_argument("--profile-warps", type=int, default=4)
    ap.add_argument("--profile-vh-bits", type=int, default=-1, help="-1: no shared-memory visited hash")
    ap.add_argument("--profile-regs", type=int, default=85)
    ap.add_argument("--profile-stage", type=int, default=-1, help="-1: vector loads; 8: TMA-staged rows")
    ap.add_argument("--phases", action="store_true", help="with --profile: per-phase cycle breakdown")
    ap.add_argument("--uneven", action="store_true",
                    help="per-query topk in {10,100} and queue in {64,128,256,512} in one launch (the default for "
                         "the deep10m workload); compares the persistent and plain schedules")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop under Poisson arrivals (request sizes log-uniform in [1,256], topk in "
                         "{10,100}, queue in {100,200,400}) against one batch_query launch per request")
    ap.add_argument("--restore", action="store_true",
                    help="HGRA snapshot to device index: streamed restore vs host reader + upload vs the reference's "
                         "restore")
    ap.add_argument("--serve-rates", default="1000,10000,50000,100000,200000")
    ap.add_argument("--serve-queries", type=int, default=20000)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    from artea_b200.graph import CompactHierarchicalGraph
    from artea_b200.router import DeviceIndex, GpuRouter

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    w, base, queries, hgra, report = wl.prepare(args.workload, args.n_base, args.n_query, log=log)
    if args.restore:
        run_restore(args, w, base, hgra, device)
        return
    metric = metric_code(w.metric)
    nq, dim, k = queries.shape[0], base.shape[1], w.topk
    graph = CompactHierarchicalGraph.from_hgra(hgra)
    index = DeviceIndex(graph, base, device=local)
    cache_dir = wl.DEFAULT_CACHE
    if args.profile:
        d_q = torch.from_numpy(queries).to(device)
        d_out = torch.empty((nq, k), dtype=torch.int64, device=device)
        r = GpuRouter(index, metric, k, args.profile_queue, mode=args.mode,
                      schedule="plain" if args.schedule == "plain" else "persistent",
                      warps_per_cta=args.profile_warps,
                      visited_hash_bits=args.profile_vh_bits if args.profile_vh_bits >= 0 else 0xFFFFFFFF,
                      register_budget=args.profile_regs, max_batch=nq,
                      stage_rows=args.profile_stage if args.profile_stage >= 0 else 0xFFFFFFFF)
        s = torch.cuda.current_stream(device)
        phases = torch.zeros((nq, 8), dtype=torch.int64, device=device) if args.phases else None
        for rep in range(2):
            if phases is not None and rep == 1:
                r.set_phase_buffer(phases)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            r.batch_query_device(d_q, nq, k, d_out, stream=s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize(device)
            log(f"profile launch: {e0.elapsed_time(e1):.3f} ms for {nq} queries")
        r.sync()
        if phases is not None:
            ph = phases.cpu().numpy().astype(np.float64)
            names = ["upper", "pop_row", "ids_visited", "distances", "merge", "tail", "total", "prefetch_hits"]
            mean = ph.mean(axis=0)
            print(json.dumps({"phase_cycles_mean": dict(zip(names, mean.tolist())),
                              "phase_share": {n: float(mean[i] / mean[6]) for i, n in enumerate(names[:6])},
                              "tuning": r.tuning()}), flush=True)
        r.close()
        index.close()
        return
    if args.serve:
        run_serving(args, w, base, queries, report, index, device, metric, cache_dir)
        index.close()
        return
    if args.uneven or w.kind == "deep":
        run_uneven(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world)
        index.close()
        return
    gt = ground_truth(index, base, queries, k, w.metric, cache_dir) if rank == 0 else None

    d_q = torch.from_numpy(queries).to(device)
    d_out = torch.empty((nq, k), dtype=torch.int64, device=device)
    d_stats = torch.zeros((nq, 8), dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)

    def make_router(L):
        return GpuRouter(index, metric, k, L, mode=args.mode, schedule=args.schedule, max_batch=nq,
                         use_graphs=not args.no_graphs)

    # Queue sweep: recall per queue size (rank 0 decides, all ranks follow).
    queues = [int(x) for x in args.queues.split(",") if x]
    sweep = []
    chosen = queues[-1]
    for L in queues:
        r = make_router(L)
        r.batch_query_device(d_q, nq, k, d_out, stream=stream.cuda_stream)
        torch.cuda.synchronize(device)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        r.batch_query_device(d_q, nq, k, d_out, stream=stream.cuda_stream)
        t1.record(stream)
        torch.cuda.synchronize(device)
        ms = t0.elapsed_time(t1)
        rec = recall(d_out.cpu().numpy().view(np.uint64), gt, k) if rank == 0 else 0.0
        sweep.append({"queue": L, "recall": round(rec, 5), "qps": nq / (ms / 1e3)})
        r.close()
    if rank == 0:
        ok = [s["queue"] for s in sweep if s["recall"] >= args.recall_target]
        chosen = ok[0] if ok else queues[-1]
    if dist is not None:
        t = torch.tensor([chosen], device=device)
        dist.broadcast(t, 0)
        chosen = int(t.item())

    router = make_router(chosen)
    # Counters for the algorithmic-byte count (untimed).
    router.batch_query_device(d_q, nq, k, d_out, d_stats=d_stats, stream=stream.cuda_stream)
    torch.cuda.synchronize(device)
    stats = d_stats.cpu().numpy().view(np.uint32)
    words = d_out.cpu().numpy().view(np.uint64)
    final_recall = recall(words, gt, k) if rank == 0 else 0.0
    alg_bytes = float(algorithmic_bytes(stats, dim, k).sum())

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        router.batch_query_device(d_q, nq, k, d_out, stream=stream.cuda_stream)
    torch.cuda.synchronize(device)

    launches0 = router.launches()
    step_ms = []
    with ClockSampler(local) as clocks:
        time.sleep(0.5)   # let nvidia-smi start sampling
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)
        t_start = time.time()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            router.batch_query_device(d_q, nq, k, d_out, stream=stream.cuda_stream)
            e1.record(stream)
            step_ms.append((e0, e1))
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()
        wall = time.perf_counter() - wall0
        clocks.mark(t_start, time.time())
        time.sleep(0.2)
    launches = router.launches() - launches0
    router.sync()
    ms = [a.elapsed_time(b) for a, b in step_ms]
    mean_ms = statistics.mean(ms)
    total_ms = sum(ms)
    if dist is not None:
        t = torch.tensor([total_ms, mean_ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, mean_ms = float(t[0]), float(t[1])
    value = world * nq * args.steps / (total_ms / 1e3)

    # End to end through the public API with host buffers.
    hq = torch.from_numpy(queries).pin_memory().numpy()
    e2e_s = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = router.batch_query(hq)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_s.append(dt)
    e2e_launches = args.steps
    e2e_mean = statistics.mean(e2e_s)
    if dist is not None:
        t = torch.tensor([e2e_mean], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_mean = float(t[0])
    e2e_value = world * nq / e2e_mean
    assert np.array_equal(out, words), "host-buffer API disagrees with the device-buffer API"

    peaks = measured_peaks()
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    traffic = profile_traffic(w.name, chosen)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peaks["source"],
                "kernel": "search_persistent_kernel" if args.schedule != "plain" else "search_plain_kernel"}

    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        baseline = cpu_baseline(hgra, base, queries, k, chosen, metric, min(args.cpu_sample, nq))

    if rank == 0:
        st = stats.astype(np.float64)
        line = {
            "metric": METRIC_NAME, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "n_base": w.n_base, "n_query": nq, "dim": dim, "metric": w.metric,
                       "topk": k, "queue": chosen, "mode": args.mode, "schedule": args.schedule,
                       "cuda_graphs": not args.no_graphs,
                       "recall_at_100": round(final_recall, 5), "parallelism": f"replicas{world}",
                       "l2": "256 MiB buffer written between timed steps (excluded from timing); "
                             "base vectors 512 MB > L2",
                       "tuning": router.tuning(),
                       "graph_levels": report.get("vertices_by_highest_level"),
                       "graph_build_s": report.get("build_s")},
            "sweep": sweep,
            "e2e": {"value": e2e_value, "unit": "queries/s",
                    "h2d_bytes_per_step": int(queries.nbytes), "d2h_bytes_per_step": int(nq * k * 8)},
            "roofline": roofline,
            "cpu_baseline": None if baseline is None else {kk: baseline[kk] for kk in
                                                           ("value", "unit", "cores", "kind", "sample", "cpu_model")},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "per_query": {"dist_evals": float(st[:, 0].mean()), "l0_rows": float(st[:, 3].mean()),
                          "upper_rows": float(st[:, 1].mean()), "bytes": alg_bytes / nq},
            "wall_s_timed_region": wall,
        }
        print(json.dumps(line), flush=True)
    router.close()
    index.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
