"""`bench.py --impl reference` on small workloads (CPU only): one JSON line
with the bench contract's keys, timed at the queue the GPU arm's recall rule
selects, the uneven per-query draws on the cosine workload, and no work on
ranks other than 0."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def run_arm(tmp_path, *extra, env=None):
    e = dict(os.environ, ARTEA_CACHE=str(tmp_path))
    e.update(env or {})
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--n-base", "3000", "--n-query", "96", "--reference-sample", "96", "--reference-select", "48",
                        *extra], cwd=str(tmp_path), env=e, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line_and_queue_rule(tmp_path):
    (line,) = run_arm(tmp_path, "--workload", "sift100k", "--queues", "100,200")
    assert KEYS <= set(line)
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    cfg = line["config"]
    assert cfg["queue"] in (100, 200) and "recall@100" in cfg["queue_selection"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    # An unreachable target falls back to the largest queue, as the GPU arm does.
    (line,) = run_arm(tmp_path, "--workload", "sift100k", "--queues", "100,200", "--recall-target", "1.01")
    assert line["config"]["queue"] == 200
    (line,) = run_arm(tmp_path, "--workload", "sift100k", "--reference-queue", "150")
    assert line["config"]["queue"] == 150


def test_reference_arm_uneven_cosine(tmp_path):
    (line,) = run_arm(tmp_path, "--workload", "deep10m")
    assert line["config"]["metric"] == "cosine" and "per query" in str(line["config"]["queue"])
    assert "groups" in line["cpu_baseline"]["sample"]


@pytest.mark.parametrize("rank", ["1"])
def test_other_ranks_print_nothing(tmp_path, rank):
    assert run_arm(tmp_path, "--workload", "sift100k", env={"RANK": rank, "WORLD_SIZE": "2"}) == []
