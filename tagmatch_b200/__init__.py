"""TagMatch subset matching on NVIDIA B200 (sm_100a).

Native engine: libtagmatch_b200.so (C ABI in include/tagmatch_b200.h).
"""
from .tagmatch import (TagMatch, balanced_partitioning, filter_from_bits, filter_from_string, filter_to_string,
                       as_filter, as_filters)
from ._native import TagMatchError, load

__all__ = ["TagMatch", "TagMatchError", "balanced_partitioning", "filter_from_bits", "filter_from_string",
           "filter_to_string", "as_filter", "as_filters", "load"]
