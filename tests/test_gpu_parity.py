"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own outputs.  Bit-exact: same multiset of keys per query for
match, same sorted unique keys for match_unique."""
import os
import subprocess
import threading

import numpy as np
import pytest

from oracle import oracle
from tagmatch_b200 import TagMatch, TagMatchError, balanced_partitioning, build, workload
from tagmatch_b200 import _native
from tagmatch_b200.tagmatch import filter_from_bits, filter_from_string
from tests.conftest import golden
from tests.helpers import (assert_same_multisets, groups_from_assignment, load_partitions_golden, read_fixtures,
                           wide_key_lists)

pytestmark = pytest.mark.gpu


def engine_with(filters, key_off, keys, max_p=65536):
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(filters, key_off, keys)
    tm.consolidate(max_p, 1)
    return tm


def check_against_oracle(f, ko, k, q, max_p, unique_too=True):
    tm = engine_with(f, ko, k, max_p)
    off, keys = tm.match_batch(q)
    ooff, okeys = oracle.match(f, ko, k, q)
    assert_same_multisets(off, keys, ooff, okeys)
    if unique_too:
        uoff, ukeys = tm.match_batch(q, unique=True)
        eoff, ekeys = oracle.match(f, ko, k, q, unique=True)
        assert np.array_equal(uoff, eoff) and np.array_equal(ukeys, ekeys)
    tm.close()


def test_small_workloads_against_reference_matcher():
    g = np.load(golden("matcher_small.npz"))
    for tag in ("a", "b"):
        f, ko, k = workload.generate_filters(int(g[f"{tag}_n"]), int(g[f"{tag}_seed"]))
        q = workload.generate_queries(int(g[f"{tag}_nq"]), f, int(g[f"{tag}_seed"]))
        for max_p in (65536, 300, 17):
            tm = engine_with(f, ko, k, max_p)
            off, keys = tm.match_batch(q)
            assert_same_multisets(off, keys, g[f"{tag}_off"], g[f"{tag}_keys"])
            uoff, ukeys = tm.match_batch(q, unique=True)
            assert np.array_equal(uoff, g[f"{tag}_uoff"]) and np.array_equal(ukeys, g[f"{tag}_ukeys"])
            tm.close()


def test_config0_against_reference_digest():
    """1M filters x 10K queries, partitions <= 65,536: digests equal the reference test_matcher's."""
    g = np.load(golden("config0_digest.npz"))
    f, ko, k, q = workload.config("config0")
    tm = engine_with(f, ko, k, 65536)
    off, keys = tm.match_batch(q)
    c, h = oracle.digest(off, keys)
    assert np.array_equal(c, g["count"]) and np.array_equal(h, g["hash"])
    uoff, ukeys = tm.match_batch(q, unique=True)
    c, h = oracle.digest(uoff, ukeys)
    assert np.array_equal(c, g["ucount"]) and np.array_equal(h, g["uhash"])
    info = tm.table_info()
    assert info["filters"] == f.shape[0] and info["partitions"] > 1
    tm.close()


@pytest.mark.parametrize("n,nq,seed,max_p", [(1, 5, 31, 1), (33, 50, 32, 1), (500, 200, 33, 7),
                                              (5000, 700, 34, 64), (50000, 300, 35, 1000), (200000, 257, 36, 65536)])
def test_random_differential(n, nq, seed, max_p):
    f, ko, k = workload.generate_filters(n, seed)
    q = workload.generate_queries(nq, f, seed)
    check_against_oracle(f, ko, k, q, max_p)


def test_partitioner_against_reference():
    gold = load_partitions_golden()
    for case in gold["fixtures"] + gold["random"]:
        f = np.asarray(case["filters"], dtype=np.uint32) if "filters" in case else \
            workload.generate_filters(case["n"], case["seed"])[0]
        part, masks, sizes = balanced_partitioning(f, case["max_p"])
        assert groups_from_assignment(part, len(sizes)) == groups_from_assignment(case["partition_of"],
                                                                                   len(case["sizes"]))
        assert sorted(tuple(int(x) for x in m) for m in masks) == sorted(tuple(m) for m in case["masks"])
        assert sorted(sizes.tolist()) == sorted(case["sizes"])


def test_partitioning_known_answers_on_gpu():
    fx = read_fixtures()
    PF = np.stack([filter_from_string(s) for s in fx["PF"]])
    PQ = np.stack([filter_from_string(s) for s in fx["PQ"]])
    part, masks, sizes = balanced_partitioning(PQ[:3], 5)
    assert len(sizes) == 1 and set(part.tolist()) == {0}
    part, masks, sizes = balanced_partitioning(PF[:3], 5)
    assert sorted(tuple(m) for m in masks.tolist()) == sorted([tuple(PF[0].tolist()), tuple((PF[1] & PF[2]).tolist())])
    part, masks, sizes = balanced_partitioning(PF, 3)
    assert len(sizes) == 5
    ml = [tuple(m) for m in masks.tolist()]
    for want, members in [(PF[3], [3]), (PF[4] & PF[9], [4, 9]), (PF[1] & PF[2] & PF[8], [1, 2, 8])]:
        pid = ml.index(tuple(want.tolist()))
        assert all(part[i] == pid for i in members)
    allf = np.concatenate([PF, PQ])
    part, masks, sizes = balanced_partitioning(allf, 4)
    for i in range(len(allf)):
        assert oracle.subset_of(masks[part[i]], allf[i])


def test_edge_cases():
    ones = np.full(6, 0xFFFFFFFF, dtype=np.uint32)
    zeros = np.zeros(6, dtype=np.uint32)
    # empty table
    tm = TagMatch()
    tm.set_persistence(False)
    tm.consolidate(1000, 1)
    off, keys = tm.match_batch(np.stack([ones, zeros]))
    assert off.tolist() == [0, 0, 0] and keys.size == 0
    # empty batch
    off, keys = tm.match_batch(np.zeros((0, 6), np.uint32))
    assert off.tolist() == [0]
    tm.close()
    # corner bits, all-ones / all-zero queries, large and extreme keys (sort path)
    fl = [filter_from_bits([0]), filter_from_bits([191]), filter_from_bits([0, 191]), filter_from_bits(range(192)),
          filter_from_bits([5, 64, 127, 128])]
    kl = [[0xFFFFFFFF, 0], [1 << 20], [7, 7 + (1 << 31)], [3], [2, 2, 2]]
    ko = np.cumsum([0] + [len(set(x)) for x in kl]).astype(np.uint32)
    kk = np.concatenate([np.unique(np.array(x, dtype=np.uint32)) for x in kl]).astype(np.uint32)
    f = np.stack(fl)
    qs = np.stack([ones, zeros, filter_from_bits([0, 191]), filter_from_bits([5, 64, 127, 128, 0]),
                   filter_from_bits(range(191))])
    for max_p in (1, 2, 1000):
        check_against_oracle(f, ko, kk, qs, max_p)
    # the all-zero filter matches every query (the reference's partitioner
    # does not terminate on it; here it is a partition with an empty mask)
    f2 = np.concatenate([f, zeros[None]])
    ko2 = np.append(ko, ko[-1] + 1).astype(np.uint32)
    kk2 = np.append(kk, 99).astype(np.uint32)
    check_against_oracle(f2, ko2, kk2, qs, 1000)
    check_against_oracle(f2, ko2, kk2, qs, 2)


def test_single_bit_and_nested_filters():
    """single_bit_filters / deepest_trie (test_tagmatch.cc:591-640) at several partition sizes."""
    ones = np.full((1, 6), 0xFFFFFFFF, dtype=np.uint32)
    single = np.stack([filter_from_bits([i]) for i in range(192)])
    nested = np.stack([filter_from_bits(range(i + 1)) for i in range(192)])
    ko = np.arange(193, dtype=np.uint32)
    kk = np.arange(192, dtype=np.uint32)
    for f in (single, nested):
        for max_p in (1, 3, 1000):
            tm = engine_with(f, ko, kk, max_p)
            off, keys = tm.match_batch(ones, unique=True)
            assert keys.tolist() == list(range(192))
            tm.close()


@pytest.mark.parametrize("max_p", [65536, 500])
def test_wide_key_counts_and_split_hit_runs(max_p):
    """Filters with 8..40 keys beside filters with 1..7, dense queries (so
    that a tile's hit mask often has several runs of adjacent bits): the
    key totals and the gather's run offsets take the slot offsets wherever
    a run or the bits below it touch a filter with 8 keys or more."""
    f, _, _ = workload.generate_filters(30000, 61)
    ko, k = wide_key_lists(f.shape[0], 61)
    q = workload.generate_queries(800, f, 61, superset_fraction=0.9)
    check_against_oracle(f, ko, k, q, max_p)


def test_many_queries_one_partition_chunks():
    """More than 256 queries routed to one partition (several chunks), and
    batches larger than the device batch limit."""
    f, ko, k = workload.generate_filters(3000, 41)
    q = workload.generate_queries(5000, f, 41, superset_fraction=0.9)
    tm = engine_with(f, ko, k, 65536)
    tm.set_batch_limit(1500)
    off, keys = tm.match_batch(q)
    ooff, okeys = oracle.match(f, ko, k, q)
    assert_same_multisets(off, keys, ooff, okeys)
    tm.close()


@pytest.mark.parametrize("nq", [1, 255, 256, 257, 767, 1023, 1024, 1025, 2049, 3333])
def test_work_item_chunk_groups(nq):
    """A work item covers up to four 256-query chunks of a partition: query
    counts on both sides of the chunk and item boundaries, the last item
    holding 1 to 4 chunks, each chunk full or partial."""
    f, ko, k = workload.generate_filters(3000, 43)
    q = workload.generate_queries(nq, f, 43 + nq, superset_fraction=0.9)
    tm = engine_with(f, ko, k, 65536)
    off, keys = tm.match_batch(q)
    ooff, okeys = oracle.match(f, ko, k, q)
    assert_same_multisets(off, keys, ooff, okeys)
    tm.close()


def test_capacity_error_reports_required_size():
    f, ko, k = workload.generate_filters(2000, 42)
    q = workload.generate_queries(100, f, 42)
    tm = engine_with(f, ko, k)
    off, keys = tm.match_batch(q)
    import ctypes
    lib = _native.load()
    out_off = np.zeros(101, dtype=np.uint64)
    small = np.zeros(1, dtype=np.uint32)
    nk = ctypes.c_uint64(0)
    st = lib.tm_match_batch(tm._h, q.ctypes.data_as(_native.u32p), 100, 0, out_off.ctypes.data_as(_native.u64p),
                            small.ctypes.data_as(_native.u32p), 1, ctypes.byref(nk))
    assert st == _native.TM_ERR_CAPACITY and nk.value == keys.size
    assert np.array_equal(out_off, off)
    tm.close()


def test_incremental_updates_and_database(tmp_path):
    """add / remove / re-consolidate through the database file (tagmatch.cc:92-142)."""
    a, b, c = filter_from_bits([1, 2]), filter_from_bits([3]), filter_from_bits([1, 2, 3])
    tm = TagMatch()
    tm.set_database_filename(str(tmp_path / "tm.db"))
    tm.add(a, [10, 11])
    tm.add(b, 20)
    tm.consolidate(1000, 1)
    q = np.stack([c])
    assert tm.match_batch(q, unique=True)[1].tolist() == [10, 11, 20]
    tm.remove(a, 10)
    tm.add(c, 30)
    tm.consolidate()
    assert tm.match_batch(q, unique=True)[1].tolist() == [11, 20, 30]
    tm.remove(b, 20)  # last key of b: b leaves the table
    tm.consolidate()
    assert tm.match_batch(q, unique=True)[1].tolist() == [11, 30]
    assert tm.table_info()["filters"] == 2
    # database file: partition_fib_entry records (u32 partition, 24-byte filter, u32 n, keys)
    raw = (tmp_path / "tm.db").read_bytes()
    assert len(raw) == (4 + 24 + 4 + 4) + (4 + 24 + 4 + 4)
    tm.clear()
    tm.consolidate()
    assert tm.match_batch(q, unique=True)[1].tolist() == []
    tm.close()


def test_async_matches_batch():
    """tm_match_async (match_handler semantics): every callback fires once,
    queries issued before start() complete after it, stop() drains."""
    f, ko, k = workload.generate_filters(20000, 43)
    q = workload.generate_queries(600, f, 43)
    tm = engine_with(f, ko, k, 4096)
    off, keys = tm.match_batch(q)
    uoff, ukeys = tm.match_batch(q, unique=True)
    got = {}
    lock = threading.Lock()

    def handler(i):
        def h(arr):
            with lock:
                assert i not in got
                got[i] = arr
        return h

    tm.set_latency_limit_ms(5)
    for i in range(300):
        tm.match(q[i], handler(i), unique=(i % 2 == 1))
    tm.start(4, 1)
    for i in range(300, 600):
        tm.match(q[i], handler(i), unique=(i % 2 == 1))
    tm.stop()
    assert len(got) == 600
    for i in range(600):
        if i % 2:
            assert np.array_equal(got[i], ukeys[uoff[i]:uoff[i + 1]])
        else:
            assert np.array_equal(np.sort(got[i]), np.sort(keys[off[i]:off[i + 1]]))
    tm.close()


def test_facade_cpp_cases(tmp_path):
    """test/test_tagmatch.cc's cases through the tagmatch.hh-compatible C++ API."""
    out = subprocess.run([build.FACADE_TEST, golden("tagmatch_fixtures.txt"), str(tmp_path / "tagmatch.db")],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 failures" in out.stdout


def test_config1_table_sampled_parity():
    """10M-filter table (seed 2): sampled queries against the oracle, and
    size-independent properties of the full result (unique is the sorted
    de-duplicated match set)."""
    f, ko, k, q = workload.config("config1", n_queries=20000)
    tm = engine_with(f, ko, k, 65536)
    off, keys = tm.match_batch(q)
    uoff, ukeys = tm.match_batch(q, unique=True)
    sample = np.arange(0, 20000, 400)
    so, sk = oracle.match(f, ko, k, q[sample])
    for j, i in enumerate(sample):
        assert np.array_equal(np.sort(keys[off[i]:off[i + 1]]), np.sort(sk[so[j]:so[j + 1]]))
    for i in range(0, 20000, 97):
        assert np.array_equal(np.unique(keys[off[i]:off[i + 1]]), ukeys[uoff[i]:uoff[i + 1]])
    tm.close()


@pytest.mark.parametrize("seg_tiles", [2048, 8192])
def test_config1_large_work_items_device_batch(seg_tiles):
    """The shapes the bench times after autotuning: the 10M-filter table,
    one device batch of 131,072 queries, 2,048 or 8,192 tiles per work item.
    Every 655th query's keys are read back from the device and compared, as
    (count, multiset hash), with the oracle's single pass over the table."""
    import torch
    from tagmatch_b200.tagmatch import read_device
    f, ko, k, q = workload.config("config1", n_queries=131072)
    tm = engine_with(f, ko, k, 65536)
    tm.set_tiles_per_item(seg_tiles)
    assert tm.get_tiles_per_item() == seg_tiles
    dq = torch.from_numpy(q.view(np.int32)).cuda()
    torch.cuda.synchronize()
    sel = np.arange(0, q.shape[0], 655)
    exp = {u: oracle.match_digest(f, ko, k, q[sel], unique=u) for u in (False, True)}
    for unique in (False, True):
        po, pk, nk = tm.match_batch_device(dq.data_ptr(), q.shape[0], unique=unique)
        off = read_device(po, q.shape[0] + 1, np.uint64)
        assert int(off[-1]) == nk
        assert np.all(off[1:] >= off[:-1])
        got_c, got_h = [], []
        for i in sel:
            keys = read_device(pk + int(off[i]) * 4, int(off[i + 1] - off[i]), np.uint32)
            if unique:
                assert np.all(keys[1:] > keys[:-1])
            c, h = oracle.digest(np.array([0, keys.size], dtype=np.uint64), keys)
            got_c.append(c[0])
            got_h.append(h[0])
        assert np.array_equal(np.array(got_c, dtype=np.uint64), exp[unique][0])
        assert np.array_equal(np.array(got_h, dtype=np.uint64), exp[unique][1])
    tm.close()


@pytest.mark.parametrize("results", [_native.TM_RESULTS_HOST, _native.TM_RESULTS_DEVICE])
@pytest.mark.parametrize("mode", [_native.TM_FLUSH_IMMEDIATE, _native.TM_FLUSH_SINGLE, _native.TM_FLUSH_FULL_OR_LATENCY])
def test_submit_requests_same_alone_and_mixed(mode, results):
    """Serving: requests of 1..700 queries, merged into shared device batches
    (or one per batch), split across batches when the batch limit is small;
    each request's result equals the same queries matched alone, with the
    keys returned in host memory or left in device memory."""
    f, ko, k = workload.generate_filters(30000, 44)
    q = workload.generate_queries(3000, f, 44)
    tm = engine_with(f, ko, k, 4096)
    rng = np.random.default_rng(5)
    reqs, at = [], 0
    while at < q.shape[0]:
        n = int(min(q.shape[0] - at, rng.integers(1, 700)))
        reqs.append((at, n, bool(rng.integers(0, 2))))
        at += n
    expect = {}
    for i, (a, n, u) in enumerate(reqs):
        expect[i] = tm.match_batch(q[a:a + n], unique=u)
    got = {}
    lock = threading.Lock()

    def handler(i):
        def h(off, keys, status):
            with lock:
                assert i not in got
                got[i] = (off, keys, status)
        return h

    tm.set_flush_mode(mode)
    tm.set_serving_results(results)
    tm.set_batch_limit(1000)  # forces merging and splitting
    tm.set_latency_limit_ms(2)
    tm.start(4, 1)
    for i, (a, n, u) in enumerate(reqs):
        tm.submit(q[a:a + n], handler(i), unique=u)
    tm.stop()
    assert len(got) == len(reqs)
    for i, (a, n, u) in enumerate(reqs):
        off, keys, status = got[i]
        eoff, ekeys = expect[i]
        assert status == 0
        assert np.array_equal(off, eoff)
        if u:
            assert np.array_equal(keys, ekeys)
        else:
            assert_same_multisets(off, keys, eoff, ekeys)
    tm.close()


def test_serve_bench_runs():
    """The serving load generator completes every request in both modes."""
    import json
    out = subprocess.run([build.SERVE_BENCH, "filters=200000", "pool=65536", "rates=20000", "seconds=1"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert {l["mode"] for l in lines} == {"plain", "continuous"}
    for l in lines:
        assert l["requests"] > 0 and l["p99_ms"] >= l["p50_ms"] > 0


def test_bulk_add_same_table_as_single_adds(tmp_path):
    """tm_add_many (sorted bulk merge at the first consolidate) builds the
    same table as one tm_add per filter (the staged update map,
    tagmatch.cc:22-34, 98-165): duplicated filters merge their keys, staged
    single adds and removals combine with the bulk ones.  The database files
    (table order, keys per filter) are byte-identical and so are the
    matches."""
    f, ko, k = workload.generate_filters(30000, 71)
    r = np.random.default_rng(4)
    dup = r.choice(f.shape[0], 3000, replace=False)
    f2 = np.concatenate([f, f[dup]])
    extra = r.integers(0, 65536, size=3000, dtype=np.uint32)
    ko2 = np.concatenate([ko, ko[-1] + np.arange(1, 3001, dtype=np.uint32)])
    k2 = np.concatenate([k, extra])
    singles = [(f[i], int(r.integers(0, 65536))) for i in r.choice(f.shape[0], 500, replace=False)]
    removes = [(f[i], int(k[ko[i]])) for i in r.choice(f.shape[0], 300, replace=False)]
    q = workload.generate_queries(2000, f, 71)
    dbs, res = [], []
    for bulk in (False, True):
        tm = TagMatch()
        db = str(tmp_path / f"bulk{int(bulk)}.db")
        tm.set_database_filename(db)
        if bulk:
            tm.add_many(f2, ko2, k2)
        else:
            for i in range(f2.shape[0]):
                tm.add(f2[i], k2[ko2[i]:ko2[i + 1]])
        for w, key in singles:
            tm.add(w, [key])
        for w, key in removes:
            tm.remove(w, key)
        tm.consolidate(4096, 1)
        res.append(tm.match_batch(q))
        tm.close()
        dbs.append(open(db, "rb").read())
    assert dbs[0] == dbs[1]
    assert_same_multisets(res[0][0], res[0][1], res[1][0], res[1][1])


@pytest.mark.parametrize("seg_tiles", [128, 4096])
def test_config2_skewed_table_sampled_parity(seg_tiles):
    """The skewed configuration at a tenth of its size: 10,000,000 filters
    with Zipf s = 1.3 tags (seed 3), so partition sizes are heavily uneven,
    and 4,096 queries at superset fractions 10%, 50% and 90%.  Every 64th
    query's keys are read back from the device and compared, as (count,
    multiset hash), with the oracle's single pass over the table; its
    match_unique keys must be the sorted de-duplicated match keys."""
    import torch
    from tagmatch_b200.tagmatch import read_device
    f, ko, k = workload.generate_filters(10_000_000, 3, zipf_s=1.3)
    tm = engine_with(f, ko, k, 65536)
    tm.set_tiles_per_item(seg_tiles)
    info = tm.table_info()
    assert info["partitions"] >= 10_000_000 // 65536
    for sup in (0.1, 0.5, 0.9):
        q = workload.generate_queries(4096, f, 3, zipf_s=1.3, superset_fraction=sup)
        sel = np.arange(0, 4096, 64)
        ec, eh = oracle.match_digest(f, ko, k, q[sel])
        dq = torch.from_numpy(q.view(np.int32)).cuda()
        torch.cuda.synchronize()
        got = {}
        for unique in (False, True):
            po, pk, nk = tm.match_batch_device(dq.data_ptr(), q.shape[0], unique=unique)
            off = read_device(po, q.shape[0] + 1, np.uint64)
            assert int(off[-1]) == nk
            got[unique] = [read_device(pk + int(off[i]) * 4, int(off[i + 1] - off[i]), np.uint32) for i in sel]
        for j in range(sel.size):
            c, h = oracle.digest(np.array([0, got[False][j].size], dtype=np.uint64), got[False][j])
            assert c[0] == ec[j] and h[0] == eh[j], (sup, int(sel[j]))
            assert np.array_equal(np.unique(got[False][j]), got[True][j])
    tm.close()


@pytest.mark.skipif(not os.environ.get("TM_SCALE_TEST"), reason="set TM_SCALE_TEST=1: 100M-filter table (minutes)")
def test_config2_scale_sampled_parity():
    """100,000,000 filters (Zipf s=1.3, seed 3): the GPU partitioner and
    table build at full size; sampled queries at superset fractions 10%, 50%
    and 90% against the oracle; match_unique equals the sorted unique match
    output; partitions respect the 65,536 maximum."""
    n = int(os.environ.get("TM_SCALE_FILTERS", "100000000"))
    f, ko, k = workload.generate_filters(n, 3, zipf_s=1.3)
    tm = engine_with(f, ko, k, 65536)
    info = tm.table_info()
    assert info["filters"] == n and info["partitions"] >= n // 65536
    for sup in (0.1, 0.5, 0.9):
        q = workload.generate_queries(4096, f, 3, zipf_s=1.3, superset_fraction=sup)
        off, keys = tm.match_batch(q)
        uoff, ukeys = tm.match_batch(q, unique=True)
        sample = np.arange(0, 4096, 256)
        so, sk = oracle.match(f, ko, k, q[sample])
        for j, i in enumerate(sample):
            assert np.array_equal(np.sort(keys[off[i]:off[i + 1]]), np.sort(sk[so[j]:so[j + 1]]))
        for i in range(0, 4096, 61):
            assert np.array_equal(np.unique(keys[off[i]:off[i + 1]]), ukeys[uoff[i]:uoff[i + 1]])
    tm.close()


def _write_fib_entries(path, f, ko, k):
    """fib_entry binary records: 24-byte filter, u32 n, n keys (fib.cc:14-21)."""
    import struct
    with open(path, "wb") as out:
        for i in range(f.shape[0]):
            b, e = int(ko[i]), int(ko[i + 1])
            out.write(f[i].astype("<u4").tobytes())
            out.write(struct.pack("<I", e - b))
            out.write(np.asarray(k[b:e], dtype="<u4").tobytes())


def test_streaming_driver_and_partition_files(tmp_path):
    """tagmatch_main.cc's flow through the C++ facade (chunked loads,
    consolidate, asynchronous match, stop drain) and the partitioning
    client's output files (partition_prefix + partition_fib_entry)."""
    import struct
    f, ko, k = workload.generate_filters(20000, 47)
    q = workload.generate_queries(2000, f, 47)
    fp, qp = tmp_path / "filters.bin", tmp_path / "queries.bin"
    _write_fib_entries(fp, f, ko, k)
    q.astype("<u4").tofile(qp)
    for unique in (0, 1):
        out = subprocess.run([build.DRIVER, f"in={fp}", f"Q={qp}", "m=4096", f"unique={unique}",
                              f"db={tmp_path / 'drv.db'}"], capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        line = [l for l in out.stdout.splitlines() if l.startswith("round=0")][0]
        fields = dict(x.split("=") for x in line.split())
        ooff, okeys = oracle.match(f, ko, k, q, unique=bool(unique))
        assert int(fields["completed"]) == q.shape[0]
        assert int(fields["keys"]) == okeys.size
    # chunked: two rounds of 10,000 filters each, each matched on its own
    out = subprocess.run([build.DRIVER, f"in={fp}", f"Q={qp}", "m=4096", "chunk=10000", f"db={tmp_path / 'drv.db'}"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rounds = [dict(x.split("=") for x in l.split()) for l in out.stdout.splitlines() if l.startswith("round=")]
    assert len(rounds) == 2
    for r, (a, b) in zip(rounds, [(0, 10000), (10000, 20000)]):
        sub_ko = (ko[a:b + 1] - ko[a]).astype(np.uint32)
        _, okeys = oracle.match(f[a:b], sub_ko, k[ko[a]:ko[b]], q)
        assert int(r["keys"]) == okeys.size
    # partition files of the reference partitioner's own seeded case
    case = load_partitions_golden()["random"][0]
    pf, pk, pkeys = workload.generate_filters(case["n"], case["seed"])
    fp2 = tmp_path / "pfilters.bin"
    _write_fib_entries(fp2, pf, pk, pkeys)
    out = subprocess.run([build.DRIVER, f"in={fp2}", f"m={case['max_p']}", f"part_out={tmp_path / 'out'}",
                          f"db={tmp_path / 'drv.db'}"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    raw = (tmp_path / "out.partitions").read_bytes()
    rec = 24 + 1 + 4 + 4
    assert len(raw) % rec == 0
    parts = []
    for i in range(len(raw) // rec):
        r = raw[i * rec:(i + 1) * rec]
        mask = np.frombuffer(r[:24], dtype="<u4")
        length, pid, size = r[24], struct.unpack("<I", r[25:29])[0], struct.unpack("<I", r[29:33])[0]
        assert length == 192 and pid == i
        parts.append((mask, size))
    fr = (tmp_path / "out.filters").read_bytes()
    part_of, pos = [], 0
    while pos < len(fr):
        pid = struct.unpack("<I", fr[pos:pos + 4])[0]
        filt = np.frombuffer(fr[pos + 4:pos + 28], dtype="<u4")
        n = struct.unpack("<I", fr[pos + 28:pos + 32])[0]
        assert oracle.subset_of(parts[pid][0], filt)
        part_of.append(pid)
        pos += 32 + 4 * n
    assert groups_from_assignment(part_of, len(parts)) == groups_from_assignment(case["partition_of"],
                                                                                 len(case["sizes"]))


def test_autotune_keeps_results():
    """tm_autotune picks tiles per work item and the batch size by timing;
    matches are the same whatever it picks."""
    f, ko, k = workload.generate_filters(100000, 48)
    q = workload.generate_queries(20000, f, 48)
    tm = engine_with(f, ko, k, 8192)
    off0, keys0 = tm.match_batch(q)
    seg, batch, qps = tm.autotune(q)
    assert seg in tuple(32 << i for i in range(9)) and batch in (8192, 16384, 20000) and qps > 0
    assert tm.get_tiles_per_item() == seg
    off1, keys1 = tm.match_batch(q)
    assert_same_multisets(off0, keys0, off1, keys1)
    tm.close()


def test_latency_limit_flushes_without_stop():
    """With a latency limit, a lone pending query completes without stop()
    (front_end.cc:563-598: queues older than the limit are flushed); with no
    limit it waits for a full batch or stop()."""
    import time
    f, ko, k = workload.generate_filters(5000, 49)
    q = workload.generate_queries(10, f, 49)
    tm = engine_with(f, ko, k, 1000)
    done = threading.Event()
    tm.set_latency_limit_ms(20)
    tm.start(2, 1)
    tm.match(q[0], lambda keys: done.set())
    assert done.wait(10.0), "latency limit did not flush the pending query"
    tm.stop()
    tm.set_latency_limit_ms(0)
    late = threading.Event()
    tm.start(2, 1)
    tm.match(q[1], lambda keys: late.set())
    time.sleep(0.3)
    assert not late.is_set()  # no limit: waits for a full batch or stop()
    tm.stop()
    assert late.is_set()
    tm.close()


def test_host_pipeline_pinned_output_and_direct_share():
    """tm_match_batch into a pinned caller buffer.  Part of each batch's keys
    is copied straight into that buffer as 32-bit values (TM_DIRECT_FRACTION),
    the rest is narrowed to 16 bits and widened by the copy threads in
    slices.  The batch limit is small, so batches outnumber the pipeline's
    lanes and the final batches shrink.  Every split, and a table whose keys
    need 32 bits, gives the same keys per query as the pageable path."""
    import ctypes

    import torch
    f, ko, k = workload.generate_filters(20000, 5)
    q = workload.generate_queries(12000, f, 5)
    assert int(k.max()) < 65536  # the 16-bit transfer applies
    for keys in (k, k + np.uint32(70000)):
        tm = engine_with(f, ko, keys, 2000)
        tm.set_batch_limit(1500)
        ref_off, ref_keys = tm.match_batch(q)
        n = q.shape[0]
        out_keys = torch.empty(max(len(ref_keys), 1), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        out_off = torch.empty(n + 1, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        lib = _native.load()
        for frac in ("0", "0.3", "1"):
            os.environ["TM_DIRECT_FRACTION"] = frac
            try:
                out_keys[:] = 0xDEADBEEF
                nk = ctypes.c_uint64(0)
                st = lib.tm_match_batch(tm._h, q.ctypes.data_as(_native.u32p), n, 0, out_off.ctypes.data_as(_native.u64p),
                                        out_keys.ctypes.data_as(_native.u32p), out_keys.size, ctypes.byref(nk))
            finally:
                del os.environ["TM_DIRECT_FRACTION"]
            assert st == 0 and nk.value == len(ref_keys)
            assert_same_multisets(out_off.copy(), out_keys[: nk.value].copy(), ref_off, ref_keys)
        tm.close()
