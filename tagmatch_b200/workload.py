"""Seeded synthetic workloads (the exact definition is in csrc/workload.cc).

Filters and queries are numpy uint32 arrays of shape [n, 6]; keys are CSR
(key_offsets [n + 1], keys).
"""
import ctypes
import os

import numpy as np

from ._native import WORKLOAD_PATH

_lib = None

CONFIGS = {
    # name: (filters, queries, seed, zipf_s, tags, superset_fraction)
    "config0": (1_000_000, 10_000, 1, 1.0, 100_000, 0.5),
    "config1": (10_000_000, 1_000_000, 2, 1.0, 100_000, 0.5),
}


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(WORKLOAD_PATH):
            raise OSError(f"{WORKLOAD_PATH} is missing: run `python -m tagmatch_b200.build`")
        lib = ctypes.CDLL(WORKLOAD_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        lib.tmw_generate_filters.restype = ctypes.c_int64
        lib.tmw_generate_filters.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double, ctypes.c_uint32,
                                             u32p, u32p, u32p]
        lib.tmw_generate_queries.restype = ctypes.c_int
        lib.tmw_generate_queries.argtypes = [ctypes.c_uint64, ctypes.c_uint64, u32p, ctypes.c_uint64,
                                             ctypes.c_double, ctypes.c_uint32, ctypes.c_double, u32p]
        lib.tmw_tag_bit.restype = ctypes.c_uint32
        lib.tmw_tag_bit.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def generate_filters(n, seed, zipf_s=1.0, tags=100_000):
    """n unique filters with 1..4 keys each: (filters [n,6], key_offsets [n+1], keys)."""
    lib = _load()
    f = np.zeros((n, 6), dtype=np.uint32)
    ko = np.zeros(n + 1, dtype=np.uint32)
    k = np.zeros(max(4 * n, 1), dtype=np.uint32)
    nk = lib.tmw_generate_filters(seed, n, zipf_s, tags, _p(f), _p(ko), _p(k))
    if nk < 0:
        raise ValueError("workload generation failed")
    return f, ko, k[:nk].copy()


def generate_queries(nq, filters, seed, zipf_s=1.0, tags=100_000, superset_fraction=0.5):
    lib = _load()
    q = np.zeros((nq, 6), dtype=np.uint32)
    filters = np.ascontiguousarray(filters, dtype=np.uint32)
    if lib.tmw_generate_queries(seed, nq, _p(filters), filters.shape[0], zipf_s, tags, superset_fraction, _p(q)) != 0:
        raise ValueError("query generation failed")
    return q


def tag_bit(tag, i):
    return _load().tmw_tag_bit(tag, i)


def config(name, n_filters=None, n_queries=None):
    """Workload of a named configuration, optionally scaled down."""
    n, nq, seed, s, tags, sup = CONFIGS[name]
    n = n_filters or n
    nq = n_queries or nq
    f, ko, k = generate_filters(n, seed, s, tags)
    q = generate_queries(nq, f, seed, s, tags, sup)
    return f, ko, k, q
