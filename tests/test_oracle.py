"""The CPU oracle, pinned against the reference's own outputs (golden
vectors produced by the reference binaries built from its sources)."""
import numpy as np
import pytest

from oracle import oracle
from tagmatch_b200 import workload
from tagmatch_b200.tagmatch import filter_from_string
from tests.conftest import golden
from tests.helpers import groups_from_assignment, load_partitions_golden, read_fixtures


def test_matcher_small_against_reference_test_matcher():
    g = np.load(golden("matcher_small.npz"))
    for tag in ("a", "b"):
        f, ko, k = workload.generate_filters(int(g[f"{tag}_n"]), int(g[f"{tag}_seed"]))
        q = workload.generate_queries(int(g[f"{tag}_nq"]), f, int(g[f"{tag}_seed"]))
        off, keys = oracle.match(f, ko, k, q, unique=False)
        # same keys in the same (table) order as the reference's test_matcher
        assert np.array_equal(off, g[f"{tag}_off"])
        assert np.array_equal(keys, g[f"{tag}_keys"])
        uoff, ukeys = oracle.match(f, ko, k, q, unique=True)
        assert np.array_equal(uoff, g[f"{tag}_uoff"])
        assert np.array_equal(ukeys, g[f"{tag}_ukeys"])


def test_cpu_backend_equals_single_pass_matcher():
    """The small-partition CPU backend restatement (back_end.cc:496-517),
    with queries routed by partition mask, gives the same per-query digests
    as the single-pass matcher over the same filters: routing by mask loses
    no match."""
    f, ko, k = workload.generate_filters(3000, 81)
    q = workload.generate_queries(400, f, 81)
    parts = oracle.partition(f, 64)
    masks = np.stack(oracle.masks_of(f, parts))
    order = np.array([i for p in parts for i in p], dtype=np.int64)
    part_off = np.zeros(len(parts) + 1, dtype=np.uint32)
    part_off[1:] = np.cumsum([len(p) for p in parts])
    fg = f[order]
    counts = (ko[1:] - ko[:-1])[order]
    kg_off = np.zeros(order.size + 1, dtype=np.uint32)
    kg_off[1:] = np.cumsum(counts)
    kg = np.concatenate([k[ko[i]:ko[i + 1]] for i in order])
    ro, rt = oracle.route(masks, q)
    c1, h1 = oracle.cpu_backend(fg, part_off, kg_off, kg, q, ro, rt)
    c2, h2 = oracle.match_digest(f, ko, k, q)
    assert np.array_equal(c1, c2) and np.array_equal(h1, h2)
    assert int(c1.sum()) > 0


def test_matcher_config0_digest():
    """1M filters x 10K queries: per-query digests equal the reference test_matcher's."""
    g = np.load(golden("config0_digest.npz"))
    f, ko, k, q = workload.config("config0")
    assert int(oracle._fin64(f.astype(np.uint64).reshape(-1)).sum(dtype=np.uint64)) == int(g["filters_hash"])
    assert int(oracle._fin64(q.astype(np.uint64).reshape(-1)).sum(dtype=np.uint64)) == int(g["queries_hash"])
    off, keys = oracle.match(f, ko, k, q, unique=False)
    c, h = oracle.digest(off, keys)
    assert np.array_equal(c, g["count"]) and np.array_equal(h, g["hash"])
    uoff, ukeys = oracle.match(f, ko, k, q, unique=True)
    c, h = oracle.digest(uoff, ukeys)
    assert np.array_equal(c, g["ucount"]) and np.array_equal(h, g["uhash"])
    # the single-pass digest matcher (the bench's parity check and CPU
    # baseline) gives the same digests on a sample of the queries
    sel = np.arange(0, q.shape[0], 25)
    c, h = oracle.match_digest(f, ko, k, q[sel])
    assert np.array_equal(c, g["count"][sel]) and np.array_equal(h, g["hash"][sel])
    c, h = oracle.match_digest(f, ko, k, q[sel], unique=True)
    assert np.array_equal(c, g["ucount"][sel]) and np.array_equal(h, g["uhash"][sel])


def test_io_known_answers():
    """test_io.cc: ASCII filter -> 24-byte binary image."""
    import json
    with open(golden("io_vectors.json")) as fh:
        cases = json.load(fh)
    assert len(cases) == 5
    for c in cases:
        w = filter_from_string(c["ascii"])
        assert list(w.astype("<u4").tobytes()) == c["bytes"]


def test_tagmatch_fixture_expectations():
    """misc_subsets / misc_subsets_Q1 expectations (test_tagmatch.cc:484-534)."""
    fx = read_fixtures()
    F = np.stack([filter_from_string(s) for s in fx["F"]])
    Q = np.stack([filter_from_string(s) for s in fx["Q"]])
    ko = np.arange(len(F) + 1, dtype=np.uint32)
    off, keys = oracle.match(F, ko, np.arange(len(F), dtype=np.uint32), Q, unique=True)
    for i in range(len(Q)):
        assert list(keys[off[i]:off[i + 1]]) == fx["E"][i]
    assert fx["E"][1] == [2]


def test_subset_and_order_semantics():
    """bitvector subset_of / operator< (bitvector.hh:282-296, 389-397)."""
    a = filter_from_string("1")           # bit 0
    b = filter_from_string("01")          # bit 1
    ab = filter_from_string("11")
    assert oracle.subset_of(a, ab) and oracle.subset_of(b, ab) and not oracle.subset_of(ab, a)
    assert oracle.subset_of(np.zeros(6, np.uint32), a)
    # bit 0 is the most significant position; a 1 there is greater
    assert oracle.filter_less(b, a) and not oracle.filter_less(a, b)
    assert oracle.filter_less(a, ab) and not oracle.filter_less(ab, ab)
    last = filter_from_string("0" * 191 + "1")
    assert oracle.filter_less(np.zeros(6, np.uint32), last) and oracle.filter_less(last, b)


def _check_partition_case(case):
    f = np.asarray(case["filters"], dtype=np.uint32) if "filters" in case else \
        workload.generate_filters(case["n"], case["seed"])[0]
    ref_groups = groups_from_assignment(case["partition_of"], len(case["sizes"]))
    ours = oracle.partition(f, case["max_p"])
    assert sorted(ours) == ref_groups
    ref_masks = sorted(tuple(m) for m in case["masks"])
    our_masks = sorted(tuple(int(x) for x in m) for m in oracle.masks_of(f, ours))
    assert our_masks == ref_masks


@pytest.mark.parametrize("i", range(4))
def test_partition_fixtures_against_reference(i):
    _check_partition_case(load_partitions_golden()["fixtures"][i])


@pytest.mark.parametrize("i", range(5))
def test_partition_random_against_reference(i):
    _check_partition_case(load_partitions_golden()["random"][i])


def test_partitioning_known_answers():
    """test_partitioning.cc:107-246 expectations, on the oracle."""
    fx = read_fixtures()
    PF = np.stack([filter_from_string(s) for s in fx["PF"]])
    PQ = np.stack([filter_from_string(s) for s in fx["PQ"]])
    assert len(oracle.partition(PQ[:3], 5)) == 1
    parts = oracle.partition(PF[:3], 5)
    masks = sorted(tuple(m) for m in oracle.masks_of(PF[:3], parts))
    assert masks == sorted([tuple(PF[0]), tuple(PF[1] & PF[2])])
    parts = oracle.partition(PF, 3)
    assert len(parts) == 5
    masks = [tuple(m) for m in oracle.masks_of(PF, parts)]
    for want, members in [(PF[3], {3}), (PF[4] & PF[9], {4, 9}), (PF[1] & PF[2] & PF[8], {1, 2, 8})]:
        assert tuple(want) in masks
        p = parts[masks.index(tuple(want))]
        assert members <= set(p)
    allf = np.concatenate([PF, PQ])
    parts = oracle.partition(allf, 4)
    assert sorted(i for p in parts for i in p) == list(range(len(allf)))
    for p, m in zip(parts, oracle.masks_of(allf, parts)):
        for i in p:
            assert oracle.subset_of(m, allf[i])
