"""Build recipe: compiles every native part in-tree.

* ``artea_b200/lib/libartea_gpu.so`` — the CUDA kernels + C-ABI, nvcc for
  sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
* ``index_build/_ref/artea_build_index`` — the reference's CPU graph builder
  (only where the reference headers are present; prebuilt copies travel).
* ``oracle/`` — the test checkers (C restatement; reference router where the
  reference headers are present).
* ``tests/cpp/_build/test_dropin`` — the C++ drop-in check (reference CPU
  router vs artea::cuda::HierarchicalGraphRouter), where the reference
  headers are present.

Run ``python -m artea_b200.build`` or call ``build()``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "artea_b200", "csrc")
LIB_DIR = os.path.join(ROOT, "artea_b200", "lib")
LIB = os.path.join(LIB_DIR, "libartea_gpu.so")
# The reference checkout: $ARTEA_REFERENCE, else a directory named "reference"
# beside this repository's root. Without one, the parts compiled from the
# reference's headers (builder, reference router, drop-in check) are skipped
# and any copies built earlier are kept.
REF = os.environ.get("ARTEA_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-pthread",
    "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cpp"))]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    deps = _sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "artea_gpu.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, *( ["-Xptxas", "-v"] if verbose else []), *_sources(), "-o", tmp]
    subprocess.run(cmd, check=True, cwd=ROOT)
    os.replace(tmp, LIB)
    return LIB


def build_make(subdir: str, with_ref: bool = True) -> None:
    args = ["make", "-C", os.path.join(ROOT, subdir)] + ([f"REF={REF}"] if with_ref else [])
    subprocess.run(args, check=True, cwd=ROOT, stdout=subprocess.DEVNULL if not os.environ.get("ARTEA_VERBOSE")
                   else None)


def build(force: bool = False) -> None:
    build_cuda(force=force)
    have_ref = os.path.isdir(os.path.join(REF, "include"))
    if not have_ref:
        print(f"[build] no reference checkout at {REF} (set ARTEA_REFERENCE): the reference router, index "
              "builder and drop-in check are not rebuilt", file=sys.stderr)
    build_make("oracle", have_ref)
    if have_ref:
        build_make("index_build")
        build_make(os.path.join("tests", "cpp"))


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
