"""mvr -- B200-native GPU multi-vector (ColBERT-style) search.

Index.load(dir, n_centroid, n_bit) / Index.search(queries, k, nprobe,
probe_topk) over libmvr's C ABI (include/mvr.h); IGPGPUBasic / IGPGPUPP
mirror the reference's method classes.
"""
from ._lib import MvrError, lib  # noqa: F401
from .index import CAND_IMPUTE, PREC_BF16, PREC_FP8, PRUNE, SEM_BASIC, SEM_PP, Index  # noqa: F401
from .igp import IGPGPUBasic, IGPGPUPP  # noqa: F401
