"""Shared helpers for the tests."""
import json
import os

import numpy as np

from tests.conftest import golden


def read_fixtures():
    """F/Q/PF/PQ filter strings and the E expectation lines of tagmatch_fixtures.txt."""
    out = {"F": {}, "Q": {}, "PF": {}, "PQ": {}, "E": {}}
    with open(golden("tagmatch_fixtures.txt")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            t = line.split()
            if t[0] == "E":
                out["E"][int(t[1])] = [int(x) for x in t[2:]]
            else:
                out[t[0]][int(t[1])] = t[2]
    return {k: [v[i] for i in sorted(v)] for k, v in out.items()}


def load_partitions_golden():
    with open(golden("partitions.json")) as f:
        return json.load(f)


def per_query_sorted(offsets, keys):
    o = np.asarray(offsets, dtype=np.int64)
    return [np.sort(keys[o[i]:o[i + 1]]) for i in range(o.size - 1)]


def assert_same_multisets(o1, k1, o2, k2):
    a = per_query_sorted(o1, k1)
    b = per_query_sorted(o2, k2)
    assert len(a) == len(b)
    for i, (x, y) in enumerate(zip(a, b)):
        assert x.size == y.size and np.array_equal(x, y), f"query {i}: {x.size} vs {y.size} keys"


def groups_from_assignment(partition_of, n_parts):
    groups = [[] for _ in range(n_parts)]
    for i, p in enumerate(partition_of):
        groups[int(p)].append(i)
    return sorted(tuple(g) for g in groups)


def wide_key_lists(n, seed):
    """Key lists for n filters in which about 10% of the filters hold 8..40
    keys (the rest 1..7), unique and sorted per filter: CSR (key_offsets,
    keys).  Counts of 8 or more take the slot-offset path of the matcher's
    per-tile key-count planes."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(1, 8, size=n)
    wide = rng.random(n) < 0.1
    counts[wide] = rng.integers(8, 41, size=int(wide.sum()))
    ko = np.zeros(n + 1, dtype=np.uint32)
    ko[1:] = np.cumsum(counts)
    keys = np.empty(int(ko[-1]), dtype=np.uint32)
    for i in range(n):
        keys[ko[i]:ko[i + 1]] = np.sort(rng.choice(65536, size=int(counts[i]), replace=False))
    return ko, keys
