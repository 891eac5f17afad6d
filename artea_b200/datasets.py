"""Seeded synthetic stand-ins for the benchmark datasets of the ARTEA query path.

The reference benchmarks on public datasets (SIFT-1M, DEEP-10M, GIST-1M) that
are not available here. These generators draw vectors with the same shapes
and value distributions (integer-valued SIFT-like, L2-normalised DEEP-like,
non-negative GIST-like) from a fixed Gaussian mixture. Every stream has its
own seed, so base, query and centre draws are reproducible one by one and
across machines running the same numpy.

Workloads (name -> shape):

* ``sift100k``: 100,000 x 128 L2, 256 centres U[0,128]^128, sigma 20,
  rounded and clipped to [0, 218]; 1,000 queries; topk 100, queue 200.
* ``sift1m``: the same generator with 1,024 centres, 1,000,000 base vectors
  and 10,000 queries; queue swept over {100, 200, 400, 800}.
* ``deep10m``: 10,000,000 x 96 cosine, 4,096 centres N(0, I), sigma 0.35,
  L2-normalised; 10,000 queries with per-query topk in {10, 100} and queue in
  {64, 128, 256, 512}.
* ``gist1m``: 1,000,000 x 960 L2, 512 centres U[0, 0.3]^960, sigma 0.05,
  clipped at 0; 1,000 queries; queue in {200, 400}; l0_min_distance 0.05.
* ``deep1m410``: deep10m's generator with 1,000,000 base vectors and 410
  centres (the 10M index's 2,439 vectors per cluster), 10,000 queries and the
  same per-query topk/queue draws: the 10M workload's search behaviour at a
  tenth of the graph build.

Any workload can be scaled down (``n_base``/``n_query`` overrides) for tests.
"""

from __future__ import annotations

import dataclasses
import hashlib
import os
import struct
from typing import Optional

import numpy as np

METRIC_L2 = "euclidean"
METRIC_COSINE = "cosine"
METRIC_DOT = "dot"


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    n_base: int
    n_query: int
    dim: int
    metric: str
    n_centres: int
    kind: str  # "sift" | "deep" | "gist"
    seed: int
    topk: int = 100
    queue: int = 200
    l0_min_distance: float = 1.0

    def scaled(self, n_base: Optional[int] = None, n_query: Optional[int] = None) -> "Workload":
        return dataclasses.replace(
            self,
            n_base=self.n_base if n_base is None else int(n_base),
            n_query=self.n_query if n_query is None else int(n_query),
            name=self.name if (n_base is None and n_query is None)
            else f"{self.name}-n{n_base or self.n_base}-q{n_query or self.n_query}",
        )


WORKLOADS = {
    "sift100k": Workload("sift100k", 100_000, 1_000, 128, METRIC_L2, 256, "sift", 1000),
    "sift1m": Workload("sift1m", 1_000_000, 10_000, 128, METRIC_L2, 1024, "sift", 1001),
    "deep10m": Workload("deep10m", 10_000_000, 10_000, 96, METRIC_COSINE, 4096, "deep", 1002,
                        topk=100, queue=512),
    "gist1m": Workload("gist1m", 1_000_000, 1_000, 960, METRIC_L2, 512, "gist", 1003,
                       queue=400, l0_min_distance=0.05),
    # deep10m's generator and queries at 1/10 of the base with 1/10 of the
    # centres: the same 2,439 vectors per cluster, so a search does what it
    # does on the 10M index, on a graph that builds in minutes.
    "deep1m410": Workload("deep1m410", 1_000_000, 10_000, 96, METRIC_COSINE, 410, "deep", 1002,
                          topk=100, queue=512),
}

_STREAM_CENTRES, _STREAM_BASE, _STREAM_QUERY, _STREAM_PARAMS = 0, 1, 2, 3
_CHUNK = 1 << 18


def _rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, stream])))


def _centres(w: Workload) -> np.ndarray:
    rng = _rng(w.seed, _STREAM_CENTRES)
    if w.kind == "sift":
        return rng.uniform(0.0, 128.0, size=(w.n_centres, w.dim)).astype(np.float32)
    if w.kind == "deep":
        return rng.standard_normal(size=(w.n_centres, w.dim), dtype=np.float32)
    if w.kind == "gist":
        return rng.uniform(0.0, 0.3, size=(w.n_centres, w.dim)).astype(np.float32)
    raise ValueError(f"unknown workload kind {w.kind!r}")


def _draw(w: Workload, centres: np.ndarray, n: int, stream: int, out: np.ndarray) -> None:
    rng = _rng(w.seed, stream)
    for lo in range(0, n, _CHUNK):
        hi = min(n, lo + _CHUNK)
        labels = rng.integers(0, w.n_centres, size=hi - lo)
        noise = rng.standard_normal(size=(hi - lo, w.dim), dtype=np.float32)
        if w.kind == "sift":
            x = centres[labels] + noise * np.float32(20.0)
            np.clip(np.rint(x), 0.0, 218.0, out=x)
        elif w.kind == "deep":
            x = centres[labels] + noise * np.float32(0.35)
            norms = np.sqrt(np.einsum("ij,ij->i", x, x, dtype=np.float32))
            norms[norms == 0] = 1.0
            x /= norms[:, None]
        else:
            x = centres[labels] + noise * np.float32(0.05)
            np.maximum(x, 0.0, out=x)
        out[lo:hi] = x


def padded_dim(dim: int) -> int:
    """Row stride in floats: the dimension rounded up to a multiple of 16.

    Mirrors the reference's SIMD padding of stored vectors
    (containers/vector_dataset.hpp:243-265): zero tail, 64-byte rows.
    """
    return (dim + 15) // 16 * 16


def generate(w: Workload) -> tuple[np.ndarray, np.ndarray]:
    """Return (base, queries) as C-contiguous float32 arrays padded to 16 columns."""
    centres = _centres(w)
    d = padded_dim(w.dim)
    base = np.zeros((w.n_base, d), dtype=np.float32)
    queries = np.zeros((w.n_query, d), dtype=np.float32)
    _draw(w, centres, w.n_base, _STREAM_BASE, base[:, : w.dim] if d != w.dim else base)
    _draw(w, centres, w.n_query, _STREAM_QUERY, queries[:, : w.dim] if d != w.dim else queries)
    return base, queries


def per_query_params(w: Workload, n_query: Optional[int] = None,
                     topk_choices=(10, 100), queue_choices=(64, 128, 256, 512)) -> tuple[np.ndarray, np.ndarray]:
    """Per-query (topk, queue) draws for uneven batches, seeded from the workload."""
    n = w.n_query if n_query is None else n_query
    rng = _rng(w.seed, _STREAM_PARAMS)
    topk = rng.choice(np.asarray(topk_choices, dtype=np.uint32), size=n)
    queue = rng.choice(np.asarray(queue_choices, dtype=np.uint32), size=n)
    queue = np.maximum(queue, topk)
    return topk.astype(np.uint32), queue.astype(np.uint32)


def fingerprint(a: np.ndarray) -> str:
    """Short content hash used to key cached graphs to the exact vectors they index."""
    h = hashlib.sha256()
    h.update(struct.pack("<QQ", *a.shape))
    h.update(np.ascontiguousarray(a).view(np.uint8).data)
    return h.hexdigest()[:16]


def write_fbin(path: str, a: np.ndarray) -> None:
    """Write ``uint32 n, uint32 d`` followed by n*d little-endian float32 values."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(struct.pack("<II", a.shape[0], a.shape[1]))
        a.tofile(f)
    os.replace(tmp, path)


def read_fbin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        n, d = struct.unpack("<II", f.read(8))
        return np.fromfile(f, dtype=np.float32, count=n * d).reshape(n, d)
