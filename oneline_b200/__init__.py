"""oneline_b200: the oneline parse-and-search hot path on NVIDIA B200 (sm_100a).

The compute runs in ``liboneline_cuda.so`` (hand-written CUDA kernels behind the
C ABI declared in ``include/oneline_cuda.h``); this package is the host-side
mirror of the reference's public API (crates oneline-core and oneline-gpu).
"""
from .core import NODE_DTYPE, NONE, FlatTree, NodeKind, TreeLinks  # noqa: F401
from ._lib import OnelineError  # noqa: F401
from .gpu import (  # noqa: F401
    MAX_GPU_INPUT_LEN,
    MAX_PATTERN_LEN,
    MAX_TREE_DEPTH,
    HIT_DTYPE,
    MAX_DICT_PATTERNS,
    MAX_PATTERNS,
    MAX_SET_PATTERN_LEN,
    MIN_SET_PATTERN_LEN,
    GpuBatch,
    GpuDocument,
    GpuParser,
    GpuPatternSet,
    GpuPipeline,
    GpuTree,
    ManyResult,
    Profile,
    QueryResult,
    SearchResult,
)
