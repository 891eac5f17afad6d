"""Workload preparation: seeded vectors plus a graph from the reference builder.

The query path searches graphs built and compacted by the reference's own CPU
builder (index_build/_ref/artea_build_index, the artea_graph factory +
compactor + HGRA snapshot). Graphs are cached by the fingerprint of the exact
vectors they index, so tests, smoke runs and benchmarks that share a workload
build it once per machine. Concurrent processes (one per GPU) serialise on a
lock file; the first builds, the others wait and reuse.
"""

from __future__ import annotations

import fcntl
import json
import os
import subprocess
import sys
import time
import zlib
from typing import Optional, Tuple

import numpy as np

from . import datasets as ds

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILDER = os.path.join(ROOT, "index_build", "_ref", "artea_build_index")
DEFAULT_CACHE = os.environ.get("ARTEA_CACHE", os.path.join(ROOT, ".cache"))
# zlib-compressed snapshots built elsewhere by the same builder for the same
# vectors (same file stem = same vector fingerprint); used instead of a build.
PREBUILT = os.path.join(ROOT, "prebuilt")

BUILD_PARAMS = dict(beta=2.0, tau_k=0.0, tau=1.5, search_nn_qs=64, loops=15, triu=4, prefill=0.4, scale=1.10,
                    shift=1.5, shuffle=1)


def graph_for(base: np.ndarray, metric: str, l0: float = 1.0, cache_dir: Optional[str] = None,
              tag: str = "graph", log=None) -> Tuple[str, dict]:
    """Path of an HGRA snapshot for ``base`` (building it if needed) and the
    builder's report (build seconds, level histogram, threads)."""
    cache_dir = cache_dir or DEFAULT_CACHE
    os.makedirs(cache_dir, exist_ok=True)
    fp = ds.fingerprint(base)
    stem = os.path.join(cache_dir, f"{tag}-{metric}-l0{l0:g}-{fp}")
    hgra, meta = stem + ".hgra", stem + ".json"
    lock = open(stem + ".lock", "w")
    try:
        fcntl.flock(lock, fcntl.LOCK_EX)
        if os.path.exists(hgra) and os.path.exists(meta):
            with open(meta) as f:
                return hgra, json.load(f)
        packed = os.path.join(PREBUILT, os.path.basename(stem))
        if os.path.exists(packed + ".hgra.z") and os.path.exists(packed + ".json"):
            _unpack(packed + ".hgra.z", hgra)
            with open(packed + ".json") as f:
                report = json.load(f)
            report["prebuilt"] = True
            with open(meta, "w") as f:
                json.dump(report, f)
            if log:
                log(f"graph restored from {packed}.hgra.z (built by the reference builder on the same vectors)")
            return hgra, report
        if not os.path.exists(BUILDER):
            raise FileNotFoundError(f"{BUILDER} is missing: build it with `make -C index_build` where the "
                                    "reference headers are available")
        fbin = stem + ".fbin"
        ds.write_fbin(fbin, base)
        args = [BUILDER, "--base", fbin, "--metric", metric, "--out", hgra + ".tmp", "--l0", str(l0)]
        for k, v in BUILD_PARAMS.items():
            args += [f"--{k.replace('_', '-')}", str(v)]
        t0 = time.time()
        if log:
            log(f"building {metric} graph over {base.shape[0]} x {base.shape[1]} with the reference builder ...")
        res = subprocess.run(args, check=True, capture_output=True, text=True)
        report = json.loads(res.stdout.strip().splitlines()[-1])
        report["wall_s"] = time.time() - t0
        os.replace(hgra + ".tmp", hgra)
        os.remove(fbin)
        with open(meta, "w") as f:
            json.dump(report, f)
        if log:
            log(f"graph built in {report['wall_s']:.1f} s: levels {report['vertices_by_highest_level']}")
        return hgra, report
    finally:
        fcntl.flock(lock, fcntl.LOCK_UN)
        lock.close()


def _unpack(src: str, dst: str) -> None:
    d = zlib.decompressobj()
    tmp = dst + ".tmp"
    with open(src, "rb") as fi, open(tmp, "wb") as fo:
        while True:
            chunk = fi.read(1 << 24)
            if not chunk:
                break
            fo.write(d.decompress(chunk))
        fo.write(d.flush())
    os.replace(tmp, dst)


def export_prebuilt(hgra: str, meta: str, level: int = 6) -> str:
    """Compress a cached snapshot into prebuilt/ under the same stem."""
    os.makedirs(PREBUILT, exist_ok=True)
    stem = os.path.join(PREBUILT, os.path.basename(hgra)[: -len(".hgra")])
    c = zlib.compressobj(level)
    with open(hgra, "rb") as fi, open(stem + ".hgra.z.tmp", "wb") as fo:
        while True:
            chunk = fi.read(1 << 24)
            if not chunk:
                break
            fo.write(c.compress(chunk))
        fo.write(c.flush())
    os.replace(stem + ".hgra.z.tmp", stem + ".hgra.z")
    with open(meta) as f, open(stem + ".json", "w") as g:
        g.write(f.read())
    return stem + ".hgra.z"


def prepare(name: str, n_base: Optional[int] = None, n_query: Optional[int] = None, cache_dir: Optional[str] = None,
            log=None):
    """(workload, base, queries, hgra_path, build_report) for a named workload."""
    w = ds.WORKLOADS[name]
    if n_base is not None or n_query is not None:
        w = w.scaled(n_base, n_query)
    base, queries = ds.generate(w)
    hgra, report = graph_for(base, w.metric, l0=w.l0_min_distance, cache_dir=cache_dir, tag=w.name, log=log)
    return w, base, queries, hgra, report


if __name__ == "__main__":
    # python -m artea_b200.workload build|export NAME [n_base n_query]
    cmd, name = sys.argv[1], sys.argv[2]
    nb = int(sys.argv[3]) if len(sys.argv) > 3 else None
    nq = int(sys.argv[4]) if len(sys.argv) > 4 else None
    w, base, queries, hgra, report = prepare(name, nb, nq, log=print)
    print(hgra, report)
    if cmd == "export":
        print(export_prebuilt(hgra, hgra[: -len(".hgra")] + ".json"))
