#!/usr/bin/env python3
"""Benchmark of the B200 hierarchical-graph router (ARTEA batch_query).

Metric: QPS at recall@100 >= 0.95 (at the recall the index gives where no
queue reaches it). One step = one batch_query of the whole query set.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default line: the 10M x 96 cosine index (seeded DEEP-like stand-in, graph from
the reference builder), 10,000 queries with per-query topk in {10, 100} and
queue in {64, 128, 256, 512} in one launch: the autotuned persistent schedule
(`value`) against the plain one-CTA-per-query launch, end to end through the
C-ABI (`e2e`), the CPU reference on the same queries with a parity check of
its words, roofline. Nested: "serving" (the serving loop on the same index
under Poisson arrivals) and "config1" (the 1M x 128 L2 index, 10,000 queries,
topk 100: queue sweep over {100, 200, 400, 800} in EXACT and FAST mode with
plain and persistent QPS, the smallest queue reaching recall 0.95 timed, with
its own parity check and CPU baseline). `--workload NAME` prints one
workload's line instead.

`value` is device time (CUDA events around each launch on its stream, inputs
already in HBM, L2 flushed between steps and excluded); `e2e` is the same
metric through the public C-ABI with host buffers inside the timed region: the
queries sit in page-locked host memory and the router returns its results in
page-locked memory, so the kernel reads the queries and writes the result rows
across the bus while it searches (pageable buffers would be staged by
copies). Multi-GPU runs are replicas (weak scaling): every rank holds the
whole index and answers its own batch; times are the max over ranks.
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
# The default line: the 10M x 96 cosine uneven batch (persistent vs plain),
# with the 1M x 128 L2 queue sweep nested under "config1" and serving points
# on the 10M index under "serving".
HEADLINE = "deep10m"
NESTED = "sift1m"
SERVE_RATES_DEFAULT = "50000,200000"
RECALL_NOTE = {
    "deep": "recall is the index's: the reference's own batch_query returns these words (parity); with 4,096 "
            "tight clusters and a hierarchy collapsed to level 0 the reference-built graph has no edges between "
            "clusters, so recall@100 >= 0.95 is out of reach for the reference's algorithm on this generator",
    "gist": "recall is the index's: the reference's own batch_query returns these words (parity)",
}


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


def profile_traffic(workload: str, tuning: dict, alg_bytes: float, queue=None):
    """DRAM read+write bytes per launch of the timed kernel from the committed
    ncu summary of this workload (profiles/search_kernel_<workload>.md), and
    where the figure came from; (None, reason) unless the summary's
    `captured_tuning:` line names the same kernel variant as the timed launch.
    The summary gives either `traffic_bytes_per_launch[_L<queue>]:` (a capture
    of this launch) or `dram_bytes_per_algorithmic_byte:` (a capture of a
    smaller case of the same kernel, scaled here by this launch's algorithmic
    bytes)."""
    p = os.path.join(ROOT, "profiles", f"search_kernel_{workload}.md")
    if not os.path.exists(p):
        return None, f"no ncu summary for {workload}"
    lines = [line.strip() for line in open(p)]
    captured = None
    for line in lines:
        if line.startswith("captured_tuning:"):
            try:
                captured = json.loads(line.split(":", 1)[1])
            except ValueError:
                captured = None
    if not captured or any(tuning.get(k) != v for k, v in captured.items()):
        return None, f"the ncu summary's kernel variant {captured} is not the timed one"

    def number(key):
        for line in lines:
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
        return None

    for key in ([f"traffic_bytes_per_launch_L{queue}:"] if queue is not None else []) + ["traffic_bytes_per_launch:"]:
        v = number(key)
        if v is not None:
            return v, f"ncu capture of this launch ({os.path.basename(p)})"
    ratio = number("dram_bytes_per_algorithmic_byte:")
    if ratio is not None:
        return ratio * alg_bytes, (f"ncu DRAM bytes per algorithmic byte of a smaller case ({os.path.basename(p)}) "
                                   "x this launch's algorithmic bytes")
    return None, "no traffic figure in the ncu summary"


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own batch_query on this host's cores.
# ---------------------------------------------------------------------------
class CpuReference:
    """The CPU side of the comparison, opened once per snapshot: the
    reference's own router (its restore of the HGRA snapshot plus
    hierarchical_graph_router_t) where it was built and the host has
    AVX-512, else the C restatement on the host reader's graph."""

    def __init__(self, hgra: str, base: np.ndarray):
        from oracle import oracle as orc
        self.orc = orc
        self.base = base
        self.ref = orc.RefRouter(hgra, base) if orc.have_ref() and host_has_avx512() else None
        if self.ref is None:
            from artea_b200.graph import CompactHierarchicalGraph
            self.graph = CompactHierarchicalGraph.from_hgra(hgra)

    def close(self):
        if self.ref is not None:
            self.ref.close()
            self.ref = None


def cpu_baseline(cpu: CpuReference, queries: np.ndarray, topk: int, queue: int, metric: int,
                 sample: int, repeats: int = 1) -> dict:
    """The reference's batch_query on this host's cores over the first `sample`
    queries; its result words are kept (key "words") for the parity check."""
    orc = cpu.orc
    base = cpu.base
    q = queries[:sample]
    threads = os.cpu_count() or 1
    words = None
    if cpu.ref is not None:
        r = cpu.ref
        r.batch_query(q[: min(256, len(q))], topk, queue, metric=metric)   # warm-up
        secs = []
        for _ in range(repeats):
            words, s = r.batch_query(q, topk, queue, metric=metric)
            secs.append(s)
        cores = int(orc.ref_lib().artea_ref_max_threads())
        kind = "reference"
    else:
        g = cpu.graph
        orc.batch_query(g, base, q[: min(256, len(q))], topk, queue, metric=metric, threads=threads)
        secs = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            words = orc.batch_query(g, base, q, topk, queue, metric=metric, threads=threads)
            secs.append(time.perf_counter() - t0)
        cores = threads
        kind = "port"
    s = statistics.mean(secs)
    return {"value": len(q) / s, "unit": "queries/s", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{len(q)} queries x {repeats} run(s) of batch_query at queue {queue}, topk {topk}",
            "seconds_per_run": s, "words": words}


INVALID_WORD = np.uint64((0x7F7FFFFF << 32) | 0x7FFFFFFF)
BASELINE_KEYS = ("value", "unit", "cores", "kind", "sample", "cpu_model")


def parity(gpu_words: np.ndarray, ref_words: np.ndarray, topk, against: str) -> dict:
    """EXACT-mode identity of the GPU's result words with the CPU reference's
    on the same queries: row i must equal the reference's k_i words, and any
    columns past k_i must hold the invalid CandidateEntry."""
    n = ref_words.shape[0]
    g = gpu_words[:n]
    ks = np.broadcast_to(np.asarray(topk), (n,))
    bad = []
    for k in np.unique(ks):
        rows = np.nonzero(ks == k)[0]
        k = int(k)
        ok = np.all(g[rows, :k] == ref_words[rows, :k], axis=1) & np.all(g[rows, k:] == INVALID_WORD, axis=1)
        bad.extend(rows[~ok].tolist())
    bad.sort()
    out = {"queries": int(n), "identical": not bad, "first_mismatch": bad[0] if bad else None,
           "rows_differing": len(bad), "against": against}
    if bad:
        i = bad[0]
        k = int(ks[i])
        out["first_mismatch_detail"] = {"gpu": [int(x) for x in g[i, :min(k, 4)]],
                                        "reference": [int(x) for x in ref_words[i, :min(k, 4)]]}
    return out


def against_name(kind: str) -> str:
    return ("the reference's batch_query (hierarchical_graph_router_t, oracle/_ref)" if kind == "reference"
            else "the C restatement of batch_query (oracle port)")


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
    """The reference's own CPU batch_query on this host's cores, on the GPU
    arm's workload, queries and per-query (topk, queue); every step is one run
    over the whole query set (or --reference-sample queries)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    name = args.workload or HEADLINE
    w, base, queries, hgra, report = wl.prepare(name, args.n_base, args.n_query, log=log)
    metric = metric_code(w.metric)
    sample = min(args.reference_sample or queries.shape[0], queries.shape[0])
    uneven = args.uneven or w.kind == "deep"
    cpu = CpuReference(hgra, base)
    if uneven:
        # The GPU arm's uneven batch: per-query topk and queue, same draws.
        topk, queue = ds.per_query_params(w, queries.shape[0])
        cfg = {"topk": "per query in {10,100}", "queue": "per query in {64,128,256,512}"}
        timed = lambda: cpu_baseline_uneven(cpu, queries, topk, queue, metric, sample)
    else:
        queue, why = reference_queue(args, w, base, queries, hgra, metric)
        cfg = {"topk": w.topk, "queue": queue, "queue_selection": why}
        timed = lambda: cpu_baseline(cpu, queries, w.topk, queue, metric, sample)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = timed()
        if i >= args.warmup:
            vals.append(info["value"])
    cpu.close()
    value = statistics.mean(vals)
    line = {"metric": METRIC_NAME, "value": value, "unit": "queries/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sample / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": w.name, "n_base": w.n_base, "n_query": sample,
                                           "dim": w.dim, "metric": w.metric, **cfg},
            "cpu_baseline": {k: info[k] for k in BASELINE_KEYS},
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


def max_over_ranks(dist, device, values):
    """Element-wise max of a list of floats over all ranks (a no-op on one rank)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def our_launches(router, launches: int) -> int:
    """Kernels of ours per router launch: the search kernel, plus the query
    order kernel when the persistent schedule ordered the batch, plus the
    full-capacity rerun kernel under the compact queue layout (launched every
    time; it exits at once when no search was handed to it)."""
    t = router.tuning()
    return launches * (1 + (1 if t.get("ordered") else 0) + (1 if t.get("queue_slack") else 0))


def bench_uneven(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world, dist):
    """One launch over queries with uneven per-query topk/queue: the persistent
    schedule (autotuned, work stealing, CUDA graphs) against the plain
    one-CTA-per-query schedule; both must return identical words, and (EXACT
    mode) the CPU reference's words."""
    import torch
    from artea_b200.router import GpuRouter
    nq, dim = queries.shape
    topk, queue = ds.per_query_params(w, nq)
    kmax = int(topk.max())
    gt = ground_truth(index, base, queries, kmax, w.metric, cache_dir) if rank == 0 else None
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
            if dist is not None:
                dist.barrier()
            t0 = time.time()
            ms = time_steps(r, d_q, nq, kmax, d_out, d_tk, d_qu, stream, args.steps, args.warmup, flush)
            if dist is not None:
                dist.barrier()
            clocks.mark(t0, time.time())
            time.sleep(0.2)
        r.sync()
        mean_ms, total_ms = max_over_ranks(dist, device, [statistics.mean(ms), sum(ms)])
        res[sched] = {"ms": mean_ms, "qps": world * nq * args.steps / (total_ms / 1e3),
                      "recall": recall(words, gt, topk) if gt is not None else None, "tuning": r.tuning(),
                      "launches": our_launches(r, r.launches() - l0 - args.warmup), "stats": stats, "words": words,
                      "clocks": clocks.summary(), "router": r}
        log(f"{sched}: {res[sched]['qps']:.0f} q/s, recall {res[sched]['recall']}, tuning {r.tuning()}")
    assert np.array_equal(res["persistent"]["words"], res["plain"]["words"]), "schedules disagree"
    p = res["persistent"]
    hq = torch.from_numpy(queries).pin_memory().numpy()   # host queries in page-locked memory, as a server holds them
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = p["router"].batch_query(hq, topk=topk, queue=queue, k_stride=kmax)
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    assert np.array_equal(out, p["words"]), "host-buffer API disagrees with the device-buffer API"
    (e2e_mean,) = max_over_ranks(dist, device, [statistics.mean(e2e)])
    alg = float(algorithmic_bytes(p["stats"], dim, topk).sum())
    peaks = measured_peaks()
    achieved = alg / (p["ms"] / 1e3) / 1e9
    baseline, par = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuReference(hgra, base)
        baseline = cpu_baseline_uneven(cpu, queries, topk, queue, metric, min(args.cpu_sample or nq, nq))
        cpu.close()
        if args.mode == "exact":
            par = parity(p["words"], baseline["words"], topk[: baseline["words"].shape[0]],
                         against_name(baseline["kind"]))
    traffic, traffic_how = profile_traffic(w.name, p["tuning"], alg)
    st = p["stats"].astype(np.float64)
    for sched in res:
        res[sched]["router"].close()
    return {
        "metric": METRIC_NAME, "value": p["qps"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": p["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "n_base": w.n_base, "n_query": nq, "dim": dim, "metric": w.metric,
                   "topk": "per query in {10,100}", "queue": "per query in {64,128,256,512}",
                   "mode": args.mode, "schedule": "persistent (autotuned, work stealing)",
                   "cuda_graphs": not args.no_graphs, "recall_at_k": p["recall"],
                   "recall_note": RECALL_NOTE.get(w.kind), "parallelism": f"replicas{world}",
                   "tuning": p["tuning"], "graph_levels": report.get("vertices_by_highest_level"),
                   "graph_build_s": report.get("build_s"),
                   "l2": "256 MiB buffer written between timed steps (excluded from timing); base vectors "
                         f"{base.nbytes / 1e9:.2f} GB"},
        "plain_one_cta_per_query": {"qps": res["plain"]["qps"], "ms_per_step": res["plain"]["ms"],
                                    "recall_at_k": res["plain"]["recall"], "tuning": res["plain"]["tuning"],
                                    "clocks": res["plain"]["clocks"]},
        "speedup_vs_plain": p["qps"] / res["plain"]["qps"],
        "parity": par,
        "e2e": {"value": world * nq / e2e_mean, "unit": "queries/s",
                "h2d_bytes_per_step": int(queries.nbytes + topk.nbytes + queue.nbytes),
                "d2h_bytes_per_step": int(nq * kmax * 8)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "traffic_source": traffic_how,
                     "algorithmic_bytes_per_launch": alg, "peak_source": peaks["source"],
                     "kernel": "search_persistent_kernel"},
        "cpu_baseline": None if baseline is None else {k: baseline[k] for k in BASELINE_KEYS},
        "gpu_launches": int(p["launches"]), "clocks": p["clocks"],
        "per_query": {"dist_evals": float(st[:, 0].mean()), "l0_rows": float(st[:, 3].mean()),
                      "upper_rows": float(st[:, 1].mean()), "bytes": alg / nq},
    }


def cpu_baseline_uneven(cpu, queries, topk, queue, metric, sample):
    """The reference router takes one (topk, queue) per instance: the sample is
    grouped by (topk, queue) and each group runs as one batch_query."""
    groups = {}
    for i in range(sample):
        groups.setdefault((int(topk[i]), int(queue[i])), []).append(i)
    total, info = 0.0, None
    words = np.full((sample, int(topk[:sample].max())), INVALID_WORD, dtype=np.uint64)
    for (k, L), idx in sorted(groups.items()):
        info = cpu_baseline(cpu, queries[idx], k, L, metric, len(idx))
        total += info["seconds_per_run"]
        words[np.asarray(idx), :k] = info["words"]
    return {"value": sample / total, "unit": "queries/s", "cores": info["cores"], "kind": info["kind"],
            "cpu_model": info["cpu_model"], "words": words, "seconds_per_run": total,
            "sample": f"{sample} queries in {len(groups)} (topk, queue) groups, one batch_query per group"}


def bench_fixed(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world, dist,
                modes=("exact",)):
    """One topk and queue for every query. Sweeps the queue sizes (recall@k,
    persistent and plain QPS, per mode), picks the smallest queue whose EXACT
    recall reaches the target, and times that queue's persistent launch:
    device steps, end to end through the host API, roofline, and the CPU
    reference on the same queries with a parity check of its words."""
    import torch
    from artea_b200.router import GpuRouter
    nq, dim, k = queries.shape[0], base.shape[1], w.topk
    gt = ground_truth(index, base, queries, k, w.metric, cache_dir) if rank == 0 else None
    d_q = torch.from_numpy(queries).to(device)
    d_out = torch.empty((nq, k), dtype=torch.int64, device=device)
    d_stats = torch.zeros((nq, 8), dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def make_router(L, mode, schedule):
        return GpuRouter(index, metric, k, L, mode=mode, schedule=schedule, max_batch=nq,
                         use_graphs=not args.no_graphs)

    queues = [int(x) for x in args.queues.split(",") if x]
    schedules = ["persistent", "plain"] if args.schedule == "auto" else [args.schedule]
    sweep = []
    for mode in modes:
        for L in queues:
            point = {"mode": mode, "queue": L}
            for sched in schedules:
                r = make_router(L, mode, sched)
                ms = time_steps(r, d_q, nq, k, d_out, None, None, stream, 3, 1, flush)
                point[f"{sched}_qps"] = nq / (statistics.median(ms) / 1e3)
                if sched == schedules[0]:
                    point["recall"] = round(recall(d_out.cpu().numpy().view(np.uint64), gt, k), 5) if rank == 0 \
                        else None
                    point["tuning"] = r.tuning()
                r.close()
            sweep.append(point)
            log(f"sweep {point}")
    exact = [p for p in sweep if p["mode"] == "exact"] or sweep
    chosen = queues[-1]
    if rank == 0:
        ok = [p["queue"] for p in exact if p["recall"] >= args.recall_target]
        chosen = ok[0] if ok else queues[-1]
    if dist is not None:
        t = torch.tensor([chosen], device=device)
        dist.broadcast(t, 0)
        chosen = int(t.item())
    mode = args.mode
    router = make_router(chosen, mode, args.schedule)
    # Counters for the algorithmic-byte count (untimed).
    router.batch_query_device(d_q, nq, k, d_out, d_stats=d_stats, stream=stream.cuda_stream)
    torch.cuda.synchronize(device)
    stats = d_stats.cpu().numpy().view(np.uint32).copy()
    words = d_out.cpu().numpy().view(np.uint64).copy()
    final_recall = recall(words, gt, k) if rank == 0 else None
    alg_bytes = float(algorithmic_bytes(stats, dim, k).sum())
    launches0 = router.launches()
    with ClockSampler(local_gpu(device)) as clocks:
        time.sleep(0.5)   # let nvidia-smi start sampling
        if dist is not None:
            dist.barrier()
        t_start = time.time()
        wall0 = time.perf_counter()
        ms = time_steps(router, d_q, nq, k, d_out, None, None, stream, args.steps, args.warmup, flush)
        if dist is not None:
            dist.barrier()
        wall = time.perf_counter() - wall0
        clocks.mark(t_start, time.time())
        time.sleep(0.2)
    launches = router.launches() - launches0 - args.warmup
    router.sync()
    mean_ms, total_ms = max_over_ranks(dist, device, [statistics.mean(ms), sum(ms)])
    value = world * nq * args.steps / (total_ms / 1e3)
    # End to end through the public API with host buffers.
    hq = torch.from_numpy(queries).pin_memory().numpy()
    e2e_s = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = router.batch_query(hq)
        if i >= args.warmup:
            e2e_s.append(time.perf_counter() - t0)
    assert np.array_equal(out, words), "host-buffer API disagrees with the device-buffer API"
    (e2e_mean,) = max_over_ranks(dist, device, [statistics.mean(e2e_s)])
    peaks = measured_peaks()
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    tuning = router.tuning()
    traffic, traffic_how = profile_traffic(w.name, tuning, alg_bytes, chosen)
    baseline, par = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuReference(hgra, base)
        baseline = cpu_baseline(cpu, queries, k, chosen, metric, min(args.cpu_sample or nq, nq))
        cpu.close()
        if mode == "exact":
            par = parity(words, baseline["words"], k, against_name(baseline["kind"]))
    n_launches = our_launches(router, launches)
    router.close()
    st = stats.astype(np.float64)
    return {
        "metric": METRIC_NAME, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "n_base": w.n_base, "n_query": nq, "dim": dim, "metric": w.metric,
                   "topk": k, "queue": chosen, "mode": mode, "schedule": args.schedule,
                   "cuda_graphs": not args.no_graphs, "recall_at_100": final_recall,
                   "recall_note": RECALL_NOTE.get(w.kind), "parallelism": f"replicas{world}",
                   "l2": "256 MiB buffer written between timed steps (excluded from timing); base vectors "
                         f"{base.nbytes / 1e9:.2f} GB",
                   "tuning": tuning, "graph_levels": report.get("vertices_by_highest_level"),
                   "graph_build_s": report.get("build_s")},
        "sweep": sweep,
        "parity": par,
        "e2e": {"value": world * nq / e2e_mean, "unit": "queries/s",
                "h2d_bytes_per_step": int(queries.nbytes), "d2h_bytes_per_step": int(nq * k * 8)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "traffic_source": traffic_how,
                     "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peaks["source"],
                     "kernel": "search_plain_kernel" if args.schedule == "plain" else "search_persistent_kernel"},
        "cpu_baseline": None if baseline is None else {kk: baseline[kk] for kk in BASELINE_KEYS},
        "gpu_launches": n_launches,
        "clocks": clocks.summary(),
        "per_query": {"dist_evals": float(st[:, 0].mean()), "l0_rows": float(st[:, 3].mean()),
                      "upper_rows": float(st[:, 1].mean()), "bytes": alg_bytes / nq},
        "wall_s_timed_region": wall,
    }


def serving_points(args, w, base, queries, index, metric, cache_dir, rates, nq):
    """The serving loop under Poisson arrivals at each offered rate: p50/p95/p99
    latency (ms), served QPS and recall@k. Requests carry 1-256 queries
    (log-uniform), topk in {10, 100}, queue in {100, 200, 400}."""
    from artea_b200.serving import Server, make_requests, run_poisson
    nq = min(nq, queries.shape[0])
    qs = queries[:nq]
    gt = ground_truth(index, base, queries, 100, w.metric, cache_dir)[:nq]
    points = []
    with Server(index, metric, max_topk=100, max_queue=400, ring_slots=16384, mode=args.mode) as srv:
        # Untimed first request: the kernel launch and module load stay out of the latencies.
        nw = min(256, nq)
        srv.wait(srv.submit(qs[:nw], topk=np.full(nw, 100, np.uint32), queue=np.full(nw, 400, np.uint32)), nw)
        for rate in rates:
            reqs = make_requests(nq, rate, seed=int(rate))
            try:
                st = run_poisson(srv, qs, reqs, 100, timeout_s=120.0)
            except TimeoutError:
                done = sum(r.n for r in reqs if r.finished is not None)
                points.append({"offered_qps": rate, "stalled": True, "queries_finished": done, "queries": nq})
                log(f"serving at {rate:.0f} q/s: STALLED after {done} of {nq} queries; later rates skipped")
                break
            order = sorted(reqs, key=lambda r: r.lo)
            words = np.vstack([r.result for r in order])
            ks = np.concatenate([r.topk for r in order])
            st["recall_at_k"] = round(recall(words, gt, ks), 5)
            st["offered_qps"] = rate
            points.append(st)
            log(f"serving at {rate:.0f} q/s: {st}")
    return points


def run_serving(args, w, base, queries, report, index, device, metric, cache_dir):
    """Serving loop under Poisson arrivals against one batch_query per request."""
    from artea_b200.router import GpuRouter
    from artea_b200.serving import make_requests, run_per_batch
    nq = min(args.serve_queries or 20000, queries.shape[0])
    qs = queries[:nq]
    rates = [float(x) for x in (args.serve_rates or "1000,10000,50000,100000,200000").split(",") if x]
    points = serving_points(args, w, base, queries, index, metric, cache_dir, rates, nq)
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
            "serving": points, "per_batch_launch": base_pts}
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
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default=None, choices=sorted(ds.WORKLOADS),
                    help="one workload's line; default: the 10M x 96 cosine uneven batch with the 1M x 128 sweep "
                         "and serving points nested")
    ap.add_argument("--n-base", type=int, default=None)
    ap.add_argument("--n-query", type=int, default=None)
    ap.add_argument("--mode", choices=("exact", "fast"), default="exact")
    ap.add_argument("--modes", default="exact,fast", help="modes of the queue sweep")
    ap.add_argument("--schedule", choices=("auto", "plain", "persistent"), default="auto")
    ap.add_argument("--queues", default=",".join(str(q) for q in DEFAULT_QUEUES))
    ap.add_argument("--recall-target", type=float, default=0.95)
    ap.add_argument("--cpu-sample", type=int, default=0, help="queries the CPU baseline runs (0: all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graphs", action="store_true", help="launch directly instead of replaying CUDA graphs")
    ap.add_argument("--no-nested", action="store_true", help="default line without the nested sweep and serving")
    ap.add_argument("--reference-queue", type=int, default=0)
    ap.add_argument("--reference-sample", type=int, default=0, help="queries per reference step (0: all)")
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
    ap.add_argument("--profile-pipeline", type=int, default=1, help="1: pipelined level-0 loop; 0: one expansion "
                                                                     "at a time")
    ap.add_argument("--profile-prefetch", type=int, default=8, help="rows loaded ahead: 8 or 16")
    ap.add_argument("--profile-slack", type=int, default=0, help="compact queue slack (0: 2L layout)")
    ap.add_argument("--profile-wpq", type=int, default=1, help="warps per query")
    ap.add_argument("--phases", action="store_true", help="with --profile: per-phase cycle breakdown")
    ap.add_argument("--profile-nq", type=int, default=0, help="with --profile: the batch's first N queries only")
    ap.add_argument("--profile-only-queue", type=int, default=0,
                    help="with --profile on per-query queues: only the queries drawn with this queue size")
    ap.add_argument("--probe", action="store_true",
                    help="subsystem probes at --profile-queue: the search traced, then the greedy descent, distance "
                         "gathers, visited set and queue replayed alone (artea_gpu_subsystem_probe)")
    ap.add_argument("--uneven", action="store_true",
                    help="per-query topk in {10,100} and queue in {64,128,256,512} in one launch (the default for "
                         "the deep10m workload); compares the persistent and plain schedules")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop under Poisson arrivals (request sizes log-uniform in [1,256], topk in "
                         "{10,100}, queue in {100,200,400}) against one batch_query launch per request")
    ap.add_argument("--restore", action="store_true",
                    help="HGRA snapshot to device index: streamed restore vs host reader + upload vs the reference's "
                         "restore")
    ap.add_argument("--serve-rates", default=None)
    ap.add_argument("--serve-queries", type=int, default=None)
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
    cache_dir = wl.DEFAULT_CACHE

    def load(name):
        w, base, queries, hgra, report = wl.prepare(name, args.n_base, args.n_query, log=log)
        graph = CompactHierarchicalGraph.from_hgra(hgra)
        index = DeviceIndex(graph, base, device=local)
        del graph
        return w, base, queries, hgra, report, index

    headline = args.workload is None
    name = HEADLINE if headline else args.workload

    if args.restore:
        w, base, queries, hgra, report = wl.prepare(name, args.n_base, args.n_query, log=log)
        run_restore(args, w, base, hgra, device)
        return
    w, base, queries, hgra, report, index = load(name)
    metric = metric_code(w.metric)
    if args.profile:
        run_profile(args, w, queries, index, metric, device)
        index.close()
        return
    if args.probe:
        import torch
        d_q = torch.from_numpy(queries).to(device)
        bits = args.profile_vh_bits if args.profile_vh_bits >= 0 else 0
        res = index.subsystem_probe(d_q, queries.shape[0], w.topk, args.profile_queue, metric, mode=args.mode,
                                    visited_hash_bits=bits)
        print(json.dumps({"workload": w.name, "queue": args.profile_queue, "visited_hash_bits": bits, **res}),
              flush=True)
        index.close()
        return
    if args.serve:
        run_serving(args, w, base, queries, report, index, device, metric, cache_dir)
        index.close()
        return
    if args.uneven or w.kind == "deep":
        line = bench_uneven(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world,
                            dist)
    else:
        line = bench_fixed(args, w, base, queries, hgra, report, index, device, metric, cache_dir, rank, world,
                           dist, modes=("exact",))
    if headline and not args.no_nested:
        rates = [float(x) for x in (args.serve_rates or SERVE_RATES_DEFAULT).split(",") if x]
        if rank == 0:
            line["serving"] = {
                "index": w.name, "request_size": "log-uniform [1,256]", "topk": "{10,100} per request",
                "queue": "{100,200,400} per request", "arrivals": "Poisson", "ring_slots": 16384,
                "points": serving_points(args, w, base, queries, index, metric, cache_dir, rates,
                                         args.serve_queries or 10000)}
        index.close()
        del base, queries
        w1, base1, queries1, hgra1, report1, index1 = load(NESTED)
        modes = tuple(m for m in args.modes.split(",") if m)
        nested = bench_fixed(args, w1, base1, queries1, hgra1, report1, index1, device, metric_code(w1.metric),
                             cache_dir, rank, world, dist, modes=modes)
        line["config1"] = {k: nested[k] for k in ("value", "unit", "ms_per_step", "config", "sweep", "parity",
                                                  "e2e", "roofline", "cpu_baseline", "gpu_launches", "clocks",
                                                  "per_query")}
        index1.close()
    else:
        index.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_profile(args, w, queries, index, metric, device):
    """One warm and one measured launch with fixed launch options (for ncu).
    The deep workload (or --uneven) takes its per-query topk and queue."""
    import torch
    from artea_b200.router import GpuRouter
    nq, k = queries.shape[0], w.topk
    topk_all, queue_all = ds.per_query_params(w, nq)
    per_query = args.uneven or w.kind == "deep"
    if args.profile_only_queue and not per_query:
        raise SystemExit("--profile-only-queue needs per-query queue sizes (a deep workload or --uneven)")
    if args.profile_only_queue:
        keep = np.nonzero(queue_all == args.profile_only_queue)[0]
        queries, topk_all, queue_all = queries[keep], topk_all[keep], queue_all[keep]
        nq = len(keep)
    if args.profile_nq:
        nq = min(nq, args.profile_nq)
        queries = np.ascontiguousarray(queries[:nq])
    d_q = torch.from_numpy(queries).to(device)
    d_tk = d_qu = None
    L = args.profile_queue
    if per_query:
        topk, queue = np.ascontiguousarray(topk_all[:nq]), np.ascontiguousarray(queue_all[:nq])
        k, L = int(topk.max()), int(queue.max())
        d_tk = torch.from_numpy(topk.view(np.int32)).to(device)
        d_qu = torch.from_numpy(queue.view(np.int32)).to(device)
    d_out = torch.empty((nq, k), dtype=torch.int64, device=device)
    r = GpuRouter(index, metric, k, L, mode=args.mode,
                  schedule="plain" if args.schedule == "plain" else "persistent",
                  warps_per_cta=args.profile_warps,
                  visited_hash_bits=args.profile_vh_bits if args.profile_vh_bits >= 0 else 0xFFFFFFFF,
                  register_budget=args.profile_regs, max_batch=nq,
                  stage_rows=args.profile_stage if args.profile_stage >= 0 else 0xFFFFFFFF,
                  pipeline=1 if args.profile_pipeline else 0xFFFFFFFF, prefetch_rows=args.profile_prefetch,
                  queue_slack=args.profile_slack or 0xFFFFFFFF, warps_per_query=args.profile_wpq)
    s = torch.cuda.current_stream(device)
    phases = torch.zeros((nq, 8), dtype=torch.int64, device=device) if args.phases else None
    d_stats = torch.zeros((nq, 8), dtype=torch.int32, device=device)
    times = []
    for rep in range(2):
        if phases is not None and rep == 1:
            r.set_phase_buffer(phases)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        r.batch_query_device(d_q, nq, k, d_out, d_topk=d_tk, d_queue=d_qu, d_stats=d_stats if rep == 0 else None,
                             stream=s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize(device)
        times.append(e0.elapsed_time(e1))
        log(f"profile launch: {times[-1]:.3f} ms for {nq} queries")
    r.sync()
    st = d_stats.cpu().numpy().view(np.uint32)
    out = {"tuning": r.tuning(), "queries": nq, "ms": times[-1],
           "per_query": {"dist_evals": float(st[:, 0].mean()), "l0_rows": float(st[:, 3].mean()),
                         "l0_rows_max": int(st[:, 3].max())}}
    if phases is not None:
        ph = phases.cpu().numpy().astype(np.float64)
        names = ["upper", "pop_row", "ids_visited", "distances", "merge", "tail", "total", "prefetch_hits"]
        mean = ph.mean(axis=0)
        out["phase_cycles_mean"] = dict(zip(names, mean.tolist()))
        out["phase_share"] = {n: float(mean[i] / mean[6]) for i, n in enumerate(names[:6])}
    print(json.dumps(out), flush=True)
    r.close()


if __name__ == "__main__":
    main()
