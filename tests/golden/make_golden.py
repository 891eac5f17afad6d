"""Generates the golden fixtures of tests/golden from the ARTEA reference itself.

Run in a container where the reference is mounted and built
(``make -C oracle`` and ``make -C index_build``):

    python tests/golden/make_golden.py

Every expected output below comes from the reference's own code: graphs from
its CPU builder (index_build/_ref/artea_build_index) and query results and
distance-call counts from its hierarchical_graph_router_t (oracle/_ref). The
hand-made graphs restate the shapes of the reference's unit tests
(unit_tests/test_router_early_stop.cpp:59-97,
unit_tests/test_compact_csr_query.cpp:20-37 and, for rows that repeat ids,
:89-146); the expected answers of the first two are also re-derived
independently (an exact sort) in the tests.
"""

from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from artea_b200 import datasets as ds  # noqa: E402
from artea_b200.graph import CompactHierarchicalGraph, INVALID_LEVEL  # noqa: E402
from oracle import oracle as orc  # noqa: E402

BUILDER = os.path.join(ROOT, "index_build", "_ref", "artea_build_index")


def early_stop_graph(top: int = 2) -> CompactHierarchicalGraph:
    """4 vertices on one axis (x0 = 12, 8, 4, 0), dim 16; L2 singleton {0};
    L1 chain 0->1->2->3; L0 complete (test_router_early_stop.cpp:69-97)."""
    hl = [top if v == 0 else min(top, 1) for v in range(4)]
    rows = []
    for v in range(4):
        r = {}
        for h in range(hl[v] + 1):
            if h == 0:
                r[0] = [o for o in range(4) if o != v]
            elif h == 1:
                r[1] = [v + 1] if (top > 0 and v < 3) else []
            else:
                r[h] = []
        rows.append(r)
    return CompactHierarchicalGraph.from_rows(4, hl, rows, entry_point_vid=0, ul_max_nbr_size=4,
                                              bl_max_nbr_size=4, top_level=top)


def early_stop_vectors() -> np.ndarray:
    v = np.zeros((4, 16), dtype=np.float32)
    v[:, 0] = [12, 8, 4, 0]
    return v


def axis_graph() -> CompactHierarchicalGraph:
    """80 vertices, dim 128, x0 = vid; vids < 40 on L1; complete rows (self
    included) on every level, as the compactor leaves the rows of
    test_compact_csr_query.cpp:24-37. Entry point: vid 19, the first vid
    closest to the top bucket's centroid (x0 = 19.5)."""
    hl = [1 if v < 40 else 0 for v in range(80)]
    rows = [{0: list(range(80)), **({1: list(range(40))} if v < 40 else {})} for v in range(80)]
    return CompactHierarchicalGraph.from_rows(80, hl, rows, entry_point_vid=19, ul_max_nbr_size=80,
                                              bl_max_nbr_size=80, top_level=1)


def axis_vectors() -> np.ndarray:
    v = np.zeros((80, 128), dtype=np.float32)
    v[:, 0] = np.arange(80, dtype=np.float32)
    return v


def axis_queries() -> np.ndarray:
    q = np.zeros((5, 128), dtype=np.float32)
    q[:, 0] = [-2.0, 12.25, 39.5, 60.75, 90.0]
    return q


REPEAT_ROW = [2, 0, 3, 3, 1, 5, 7, 5, 4, 6, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18]


def repeats_graph(n: int = 320, seed: int = 23):
    """Rows that name ids more than once and ids already visited, restating at
    graph scale what unit_tests/test_compact_csr_query.cpp:89-146 pins for
    process_prefetched_neighbors: a later occurrence of an id in the row, and
    an id visited before the row is read, are skipped; ids are marked visited
    when collected. Vertex 20's level-0 row is that test's row; 0, 1 and 20
    open the entry vertex's level-0 row. Other level-0 rows are each vertex's
    nearest vertices with repeats, the vertex itself and the entry point mixed
    in; some are longer than 64 ids (bl 96), so the collect loop takes them in
    several chunks. Level-1 rows repeat ids too. Integer-valued vectors give
    many equal distances. Returns (graph, base, queries)."""
    rng = np.random.default_rng(seed)
    dim = 16
    base = rng.integers(0, 6, size=(n, dim)).astype(np.float32)
    queries = rng.integers(0, 6, size=(40, dim)).astype(np.float32)
    entry = 21
    hl = [0] * n
    lvl1 = sorted(set([entry, 20] + rng.choice(n, 30, replace=False).tolist()))
    for v in lvl1:
        hl[v] = 1
    d2 = ((base[:, None, :] - base[None, :, :]) ** 2).sum(-1)
    rows = []
    for v in range(n):
        r = {}
        order = [int(u) for u in np.argsort(d2[v], kind="stable") if u != v]
        k = int(rng.integers(6, 40))
        row = order[:k]
        for _ in range(int(rng.integers(1, 12))):                    # repeats, adjacent or later
            pos = int(rng.integers(0, len(row) + 1))
            row.insert(pos, row[int(rng.integers(0, len(row)))])
        if rng.random() < 0.5:
            row.insert(int(rng.integers(0, len(row) + 1)), v)          # the vertex itself (visited)
        if rng.random() < 0.5:
            row.insert(int(rng.integers(0, len(row) + 1)), entry)      # the entry point
        if rng.random() < 0.15:
            row = (row * 3)[: int(rng.integers(65, 97))]               # longer than 64, repeats
        r[0] = row[:96]
        if hl[v] == 1:
            others = [u for u in lvl1 if u != v]
            up = [int(u) for u in rng.choice(others, int(rng.integers(3, 12)), replace=False)]
            up = up + up[: int(rng.integers(0, len(up) + 1))]
            rng.shuffle(up)
            r[1] = up[:40]
        rows.append(r)
    rows[20][0] = list(REPEAT_ROW)
    rows[entry][0] = [0, 1, 20] + [u for u in rows[entry][0] if u not in (0, 1, 20)][:40]
    g = CompactHierarchicalGraph.from_rows(n, hl, rows, entry_point_vid=entry, ul_max_nbr_size=40,
                                           bl_max_nbr_size=96, top_level=1)
    return g, base, queries


def build_graph(base: np.ndarray, metric: str, workdir: str, **params) -> str:
    fbin = os.path.join(workdir, "base.fbin")
    out = os.path.join(workdir, "graph.hgra")
    ds.write_fbin(fbin, base)
    args = [BUILDER, "--base", fbin, "--metric", metric, "--out", out]
    for k, v in params.items():
        args += [f"--{k.replace('_', '-')}", str(v)]
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)
    return out


def ref_results(hgra: str, base: np.ndarray, queries: np.ndarray, topk: int, queue: int, metric: int,
                l0_only: bool = False):
    r = orc.RefRouter(hgra, base)
    words, _ = r.batch_query(queries, topk, queue, metric=metric, l0_only=l0_only, threads=4)
    _, _, calls = r.batch_query(queries, topk, queue, metric=metric, l0_only=l0_only, count_distances=True)
    r.close()
    return words, calls


def save_case(name: str, graph: CompactHierarchicalGraph, base: np.ndarray, queries: np.ndarray, metric: int,
              topk: int, queues, base_dtype=np.float32, l0_only=False) -> None:
    with tempfile.TemporaryDirectory() as tmp:
        hgra = os.path.join(tmp, "g.hgra")
        graph.to_hgra(hgra)
        payload = {
            "hgra": np.frombuffer(open(hgra, "rb").read(), dtype=np.uint8),
            "base": base.astype(base_dtype),
            "queries": queries.astype(np.float32),
            "metric": np.int32(metric),
            "topk": np.int32(topk),
            "queues": np.asarray(queues, dtype=np.int32),
        }
        for L in queues:
            words, calls = ref_results(hgra, base, queries, topk, L, metric)
            payload[f"words_L{L}"] = words
            payload[f"calls_L{L}"] = calls
            if l0_only:
                w0, c0 = ref_results(hgra, base, queries, topk, L, metric, l0_only=True)
                payload[f"l0_words_L{L}"] = w0
                payload[f"l0_calls_L{L}"] = c0
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **payload)
    print(name, {k: v.shape for k, v in payload.items()})


def built_case(name: str, workload: str, n_base: int, n_query: int, metric_build: str, metric: int, topk: int,
               queues, quantize_u8: bool = False, **params) -> None:
    w = ds.WORKLOADS[workload].scaled(n_base, n_query)
    base, queries = ds.generate(w)
    with tempfile.TemporaryDirectory() as tmp:
        hgra = build_graph(base, metric_build, tmp, **params)
        graph = CompactHierarchicalGraph.from_hgra(hgra)
    save_case(name, graph, base, queries, metric, topk, queues,
              base_dtype=np.uint8 if quantize_u8 else np.float32, l0_only=True)


def graph_of(path: str) -> CompactHierarchicalGraph:
    with tempfile.TemporaryDirectory() as tmp:
        hgra = os.path.join(tmp, "g.hgra")
        with open(hgra, "wb") as f:
            f.write(np.load(path)["hgra"].tobytes())
        return CompactHierarchicalGraph.from_hgra(hgra)


def entry_threshold(path: str, quantile: float) -> float:
    """A configuration-unit threshold that stops some walks early: the given
    quantile of the query-to-entry-point distances (square-rooted for L2^2)."""
    d = np.load(path)
    g = graph_of(path)
    base = d["base"].astype(np.float32)
    metric = int(d["metric"])
    ent = np.array([orc.ref_distance(metric, q, base[g.entry_point_vid]) for q in d["queries"]], dtype=np.float64)
    if metric == 0:
        ent = np.sqrt(ent)
    return float(np.quantile(ent, quantile))


def add_early_stop(name: str, configs) -> None:
    """Adds, for each per-level configuration threshold array, the reference's
    batch_query<false, true> words and per-query distance calls at every queue
    size of the case: keys es_cfg{i}, es_words{i}_L{L}, es_calls{i}_L{L}."""
    path = os.path.join(HERE, f"{name}.npz")
    d = dict(np.load(path))
    for key in [k for k in d if k.startswith("es_")]:
        del d[key]
    with tempfile.TemporaryDirectory() as tmp:
        hgra = os.path.join(tmp, "g.hgra")
        with open(hgra, "wb") as f:
            f.write(d["hgra"].tobytes())
        base = d["base"].astype(np.float32)
        r = orc.RefRouter(hgra, base)
        for i, cfg in enumerate(configs):
            cfg = np.asarray(cfg, dtype=np.float32)
            d[f"es_cfg{i}"] = cfg
            for L in d["queues"]:
                words, calls = r.batch_query_early_stop(d["queries"], int(d["topk"]), int(L), cfg,
                                                        metric=int(d["metric"]), count_distances=True)
                d[f"es_words{i}_L{L}"] = words
                d[f"es_calls{i}_L{L}"] = calls
        r.close()
    np.savez_compressed(path, **d)
    print(name, "early stop:", len(configs), "threshold sets")


def early_stop_fixtures() -> None:
    # test_router_early_stop.cpp:52-53: theta=1 gives gamma=4, T_1=8, T_2=16.
    add_early_stop("early_stop_top2", [[0, 8, 16], [0, 100, 100], [0, 4, 4]])
    add_early_stop("early_stop_sqr", [[0, 8, 16], [0, 100, 100], [0, 4, 4]])
    for name in ("sift2k", "gist400"):
        path = os.path.join(HERE, f"{name}.npz")
        top = graph_of(path).top_occupied_level_id()
        add_early_stop(name, [[0.0] + [entry_threshold(path, q)] * top for q in (0.2, 0.5)])


def add_bruteforce(name: str, topks, subset_seed: int = 5) -> None:
    """Adds the reference bruteforce_router_t's batch_query words for each topk
    (bf_k{k}) and, over a seeded subset of the vectors, its subset overload
    (bf_subset, bf_sub_k{k})."""
    path = os.path.join(HERE, f"{name}.npz")
    d = dict(np.load(path))
    for key in [k for k in d if k.startswith("bf_")]:
        del d[key]
    base = d["base"].astype(np.float32)
    rng = np.random.default_rng(subset_seed)
    subset = np.sort(rng.choice(base.shape[0], size=max(1, base.shape[0] // 3), replace=False)).astype(np.uint32)
    with tempfile.TemporaryDirectory() as tmp:
        hgra = os.path.join(tmp, "g.hgra")
        with open(hgra, "wb") as f:
            f.write(d["hgra"].tobytes())
        r = orc.RefRouter(hgra, base)
        d["bf_subset"] = subset
        for k in topks:
            d[f"bf_k{k}"] = r.bruteforce(d["queries"], k, metric=int(d["metric"]))
            d[f"bf_sub_k{k}"] = r.bruteforce(d["queries"], k, metric=int(d["metric"]), subset=subset)
        r.close()
    np.savez_compressed(path, **d)
    print(name, "bruteforce:", list(topks))


def bruteforce_fixtures() -> None:
    add_bruteforce("early_stop_top2", [1, 3, 10])      # 4 vectors: topk 10 pads
    add_bruteforce("axis80", [10, 100])                 # tied distances
    add_bruteforce("sift2k", [10, 100])
    add_bruteforce("deep1k_cos", [10, 64])
    add_bruteforce("gist400", [10, 50])


def main() -> None:
    if "--bruteforce-only" in sys.argv:
        bruteforce_fixtures()
        return
    if "--early-stop-only" in sys.argv:
        early_stop_fixtures()
        return
    if "--repeats-only" in sys.argv:
        g, base, queries = repeats_graph()
        save_case("repeats", g, base, queries, metric=0, topk=10, queues=[10, 32, 100], l0_only=True)
        return
    # Hand-made graphs from the reference unit tests.
    for top in (0, 2):
        save_case(f"early_stop_top{top}", early_stop_graph(top), early_stop_vectors(), early_stop_vectors(),
                  metric=1, topk=1, queues=[4])
    save_case("early_stop_sqr", early_stop_graph(2), early_stop_vectors(), early_stop_vectors(), metric=0, topk=1,
              queues=[4])
    save_case("axis80", axis_graph(), axis_vectors(), axis_queries(), metric=0, topk=10, queues=[80, 10, 16])
    # Graphs from the reference builder on seeded synthetic data.
    built_case("sift2k", "sift100k", 2000, 64, "euclidean", 0, 10, [10, 32, 100], quantize_u8=True)
    built_case("deep1k_cos", "deep10m", 1000, 48, "cosine", 2, 10, [16, 64])
    built_case("gist400", "gist1m", 400, 24, "euclidean", 0, 10, [20, 50], l0=0.05)
    g, base, queries = repeats_graph()
    save_case("repeats", g, base, queries, metric=0, topk=10, queues=[10, 32, 100], l0_only=True)
    early_stop_fixtures()
    bruteforce_fixtures()


if __name__ == "__main__":
    main()
