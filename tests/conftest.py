"""Shared test helpers. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["early_stop_top0", "early_stop_top2", "early_stop_sqr", "axis80", "sift2k", "deep1k_cos", "gist400",
                "repeats"]
EARLY_STOP_CASES = ["early_stop_top2", "early_stop_sqr", "sift2k", "gist400"]
BUILDER = os.path.join(ROOT, "index_build", "_ref", "artea_build_index")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


class Case:
    """One golden fixture: graph (from its HGRA bytes), vectors, queries and the
    reference router's outputs per queue size."""

    def __init__(self, name):
        from artea_b200.graph import CompactHierarchicalGraph
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.base = z["base"].astype(np.float32)
        self.queries = z["queries"]
        self.metric = int(z["metric"])
        self.topk = int(z["topk"])
        self.queues = [int(x) for x in z["queues"]]
        self.words = {L: z[f"words_L{L}"] for L in self.queues}
        self.calls = {L: z[f"calls_L{L}"] for L in self.queues}
        self.l0_words = {L: z[f"l0_words_L{L}"] for L in self.queues if f"l0_words_L{L}" in z}
        self.l0_calls = {L: z[f"l0_calls_L{L}"] for L in self.queues if f"l0_calls_L{L}" in z}
        # enable_early_stop=true outputs: per threshold set i, the configuration
        # thresholds and the reference's words / distance calls per queue size.
        self.es = []
        i = 0
        while f"es_cfg{i}" in z:
            self.es.append((z[f"es_cfg{i}"], {L: z[f"es_words{i}_L{L}"] for L in self.queues},
                            {L: z[f"es_calls{i}_L{L}"] for L in self.queues}))
            i += 1
        fd, path = tempfile.mkstemp(suffix=".hgra")
        with os.fdopen(fd, "wb") as f:
            f.write(z["hgra"].tobytes())
        self.hgra_path = path
        self.graph = CompactHierarchicalGraph.from_hgra(path)


_cases = {}


def golden_case(name) -> Case:
    if name not in _cases:
        _cases[name] = Case(name)
    return _cases[name]


def build_graph(base, metric, workdir, **params):
    """Runs the reference builder (prebuilt binary) on base; returns the HGRA path."""
    import subprocess
    from artea_b200 import datasets as ds
    fbin = os.path.join(workdir, "base.fbin")
    out = os.path.join(workdir, "graph.hgra")
    ds.write_fbin(fbin, base)
    args = [BUILDER, "--base", fbin, "--metric", metric, "--out", out]
    for k, v in params.items():
        args += [f"--{k.replace('_', '-')}", str(v)]
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)
    return out


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def assert_same_knn(got: np.ndarray, want: np.ndarray, what: str = "") -> None:
    """Rows of CandidateEntry words that must agree except for the order of
    entries at equal distance (the reference's partial_sort leaves it open):
    identical distance bits position by position, identical id sets per
    distance value, identical words everywhere else."""
    assert got.shape == want.shape, (got.shape, want.shape, what)
    gd = (got >> np.uint64(32)).astype(np.uint32)
    wd = (want >> np.uint64(32)).astype(np.uint32)
    np.testing.assert_array_equal(gd, wd, err_msg=f"{what}: distances")
    for i in range(got.shape[0]):
        if np.array_equal(got[i], want[i]):
            continue
        for dv in np.unique(wd[i]):
            g = np.sort(got[i][gd[i] == dv] & np.uint64(0xFFFFFFFF))
            w = np.sort(want[i][wd[i] == dv] & np.uint64(0xFFFFFFFF))
            if np.array_equal(g, w):
                continue
            # A tie group cut by the k boundary may hold different members.
            at_end = gd[i][-1] == dv
            assert at_end and g.size == w.size, f"{what}: row {i} ids differ at distance bits {dv:#x}"


def big_snapshot(path, n=700_000, seed=7):
    """~25 M words of vertex records of uneven length (empty rows included),
    so records cross the 8 M-word staging chunks at every kind of position; a
    few thousand vertices sit on levels 1 and 2 and 500 are unassigned."""
    rng = np.random.default_rng(seed)
    bl, ul = 64, 32
    hl = np.zeros(n, np.int64)
    hl[rng.choice(n, 3000, replace=False)] = 1
    hl[rng.choice(np.nonzero(hl == 1)[0], 40, replace=False)] = 2
    entry = int(np.nonzero(hl == 2)[0][0])
    unassigned = np.zeros(n, bool)
    unassigned[rng.choice(np.nonzero(hl == 0)[0], 500, replace=False)] = True
    valid0 = np.nonzero(~unassigned)[0].astype(np.uint32)
    lvl1 = np.nonzero(hl >= 1)[0]
    lvl2 = np.nonzero(hl == 2)[0]
    plain = (hl == 0) & ~unassigned
    cnt0 = rng.integers(0, bl + 1, n)
    special = {}
    for v in np.nonzero(hl >= 1)[0]:
        rec = [int(hl[v])]
        for lvl in range(int(hl[v]), -1, -1):
            if lvl == 0:
                ids = valid0[rng.integers(0, valid0.size, int(cnt0[v]))]
            else:
                pool = lvl2 if lvl == 2 else lvl1
                ids = rng.choice(pool, int(rng.integers(0, min(ul, pool.size) + 1)), replace=False)
            rec += [len(ids)] + [int(x) for x in ids]
        special[int(v)] = np.array(rec, np.uint32)
    rec_len = np.where(unassigned, 1, 2 + cnt0)
    for v, r in special.items():
        rec_len[v] = r.size
    start = 7 + np.concatenate([[0], np.cumsum(rec_len)[:-1]])
    words = np.zeros(7 + int(rec_len.sum()), np.uint32)
    words[:7] = [0x48475241, 1, n, 2, ul, bl, entry]
    words[start[unassigned]] = 0xFFFFFFFF
    pv = np.nonzero(plain)[0]
    words[start[pv]] = 0
    words[start[pv] + 1] = cnt0[pv]
    c = cnt0[pv]
    first = np.repeat(start[pv] + 2, c)
    within = np.arange(int(c.sum())) - np.repeat(np.concatenate([[0], np.cumsum(c)[:-1]]), c)
    words[first + within] = valid0[rng.integers(0, valid0.size, int(c.sum()))]
    for v, r in special.items():
        words[start[v]:start[v] + r.size] = r
    words.tofile(path)
    return rng.standard_normal((n, 16)).astype(np.float32)
