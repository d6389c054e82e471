"""csaw: B200-native graph sampling and random walks (C-SAW operator surface).

The compute path is libcsaw_b200.so (hand-written sm_100a CUDA behind a C
ABI, include/csaw.h); this package is its host-side binding.
"""
from . import graphgen
from ._lib import (BIAS_DEGREE, BIAS_EDGE_WEIGHT, BIAS_HOOK, BIAS_UNBIASED, MODE_MDRW, MODE_NEIGHBOR,
                   MODE_WALK, SCHED_BATCHED, SCHED_LEARNED, SCHED_PLAIN, CsawError, lib)
from .sampler import Arguments, BatchJob, Graph, Sampler, Server, StreamGraph, edge_bound, make_params

__all__ = [
    "graphgen", "lib", "Graph", "StreamGraph", "Server", "Sampler", "Arguments", "BatchJob", "make_params", "edge_bound", "CsawError",
    "MODE_NEIGHBOR", "MODE_WALK", "MODE_MDRW", "BIAS_UNBIASED", "BIAS_DEGREE", "BIAS_EDGE_WEIGHT",
    "BIAS_HOOK", "SCHED_PLAIN", "SCHED_BATCHED", "SCHED_LEARNED",
]
