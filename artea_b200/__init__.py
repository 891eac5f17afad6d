"""artea_b200 — B200 (sm_100a) query path for ARTEA compact hierarchical graphs.

A drop-in for the reference router's batch_query
(hierarchical_graph_router_t<Metric, Dim>): the graph (built and compacted by
the reference's CPU builder) and its FP32 vectors are uploaded once; queries
run in hand-written CUDA kernels behind the C-ABI of include/artea_gpu.h.
"""
from .graph import CompactHierarchicalGraph  # noqa: F401
from .router import (BruteforceRouter, DeviceIndex, GpuRouter, HierarchicalGraphRouter, entry_dists,  # noqa: F401
                     entry_vids)

__all__ = ["BruteforceRouter", "CompactHierarchicalGraph", "DeviceIndex", "GpuRouter", "HierarchicalGraphRouter",
           "entry_vids", "entry_dists"]
