"""Python side of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

* `match` -- the C restatement of the reference's sequential matcher
  (oracle.c; test_matcher.cc:74-81 + tagmatch_query.hh:99-119).
* `partition` -- the C restatement of partitioning.cc.
* `run_ref_matcher` / `run_ref_partition` -- the reference's own code, built
  from its sources into oracle/_ref by oracle/Makefile (only where the
  reference sources exist; the GPU box uses whatever was prebuilt).
* `digest` -- order-independent per-query multiset hashes for comparing
  result sets of any size.
"""
import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_MATCHER = os.path.join(HERE, "_ref", "test_matcher")
REF_PARTITION = os.path.join(HERE, "_ref", "ref_partition")
GOLDEN = np.uint64(0x9E3779B97F4A7C15)

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        lib.oracle_count.argtypes = [u32p, ctypes.c_uint64, u32p, u32p, u32p, ctypes.c_uint64, u64p, ctypes.c_int]
        lib.oracle_fill.argtypes = [u32p, ctypes.c_uint64, u32p, u32p, u32p, ctypes.c_uint64, ctypes.c_int, u64p, u32p,
                                    u64p, ctypes.c_int]
        lib.oracle_match_digest.argtypes = [u32p, ctypes.c_uint64, u32p, u32p, u32p, ctypes.c_uint64, ctypes.c_int,
                                            u64p, u64p, ctypes.c_int]
        lib.oracle_cpu_backend.argtypes = [u32p, u32p, ctypes.c_uint64, u32p, u32p, u32p, ctypes.c_uint64, u32p, u32p,
                                           u64p, u64p, ctypes.c_int]
        lib.oracle_partition.restype = ctypes.c_int64
        lib.oracle_partition.argtypes = [u32p, ctypes.c_uint32, ctypes.c_uint32, u32p, u32p, u32p, ctypes.c_uint64]
        lib.oracle_subset_of.argtypes = [u32p, u32p]
        lib.oracle_filter_less.argtypes = [u32p, u32p]
        _lib = lib
    return _lib


def _p32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _p64(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def match(filters, key_off, keys, queries, unique=False, threads=None):
    """Returns (offsets [nq + 1], keys) like the engine's tm_match_batch."""
    lib = _load()
    threads = threads or os.cpu_count() or 1
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    q = np.ascontiguousarray(queries, dtype=np.uint32).reshape(-1, 6)
    ko = np.ascontiguousarray(key_off, dtype=np.uint32)
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    if k.size == 0:
        k = np.zeros(1, dtype=np.uint32)
    nq = q.shape[0]
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    lib.oracle_count(_p32(f), f.shape[0], _p32(ko), _p32(k), _p32(q), nq, _p64(counts), threads)
    offs = np.zeros(nq + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(counts[:nq])
    out = np.zeros(max(int(offs[-1]), 1), dtype=np.uint32)
    final = np.zeros(max(nq, 1), dtype=np.uint64)
    lib.oracle_fill(_p32(f), f.shape[0], _p32(ko), _p32(k), _p32(q), nq, 1 if unique else 0, _p64(offs), _p32(out),
                    _p64(final), threads)
    if not unique:
        return offs, out[: int(offs[-1])]
    uo = np.zeros(nq + 1, dtype=np.uint64)
    uo[1:] = np.cumsum(final[:nq])
    res = np.concatenate([out[int(offs[i]): int(offs[i]) + int(final[i])] for i in range(nq)]) if nq else out[:0]
    return uo, res.astype(np.uint32)


def match_digest(filters, key_off, keys, queries, unique=False, threads=None):
    """One scan of the table per query, as test_matcher.cc:74-81 does, with
    each query's keys reduced to `digest`'s (count, multiset hash)."""
    lib = _load()
    threads = threads or os.cpu_count() or 1
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    q = np.ascontiguousarray(queries, dtype=np.uint32).reshape(-1, 6)
    ko = np.ascontiguousarray(key_off, dtype=np.uint32)
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    if k.size == 0:
        k = np.zeros(1, dtype=np.uint32)
    nq = q.shape[0]
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    hashes = np.zeros(max(nq, 1), dtype=np.uint64)
    lib.oracle_match_digest(_p32(f), f.shape[0], _p32(ko), _p32(k), _p32(q), nq, 1 if unique else 0, _p64(counts),
                            _p64(hashes), threads)
    return counts[:nq], hashes[:nq]


def route(masks, queries, chunk=4096):
    """Queries routed to each partition (mask subset of the query): CSR
    (route_off [P + 1] uint32, routed query indices uint32)."""
    m = np.ascontiguousarray(masks, dtype=np.uint32).reshape(-1, 6)
    q = np.ascontiguousarray(queries, dtype=np.uint32).reshape(-1, 6)
    lists = [[] for _ in range(m.shape[0])]
    for q0 in range(0, q.shape[0], chunk):
        qq = q[q0:q0 + chunk]
        ok = np.ones((m.shape[0], qq.shape[0]), dtype=bool)
        for w in range(6):
            ok &= (m[:, w][:, None] & ~qq[:, w][None, :]) == 0
        for p, qi in zip(*np.nonzero(ok)):
            lists[p].append(q0 + qi)
    off = np.zeros(m.shape[0] + 1, dtype=np.uint32)
    off[1:] = np.cumsum([len(x) for x in lists])
    routed = np.array([i for x in lists for i in x], dtype=np.uint32)
    return off, routed


def cpu_backend(filters, part_off, key_off, keys, queries, route_off, routed, threads=None):
    """The reference's small-partition CPU backend (back_end.cc:496-517):
    per partition, every filter against every routed query.  filters are
    grouped by partition (part_off); returns digest (count, hash) arrays."""
    lib = _load()
    threads = threads or os.cpu_count() or 1
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    po = np.ascontiguousarray(part_off, dtype=np.uint32)
    ko = np.ascontiguousarray(key_off, dtype=np.uint32)
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    if k.size == 0:
        k = np.zeros(1, dtype=np.uint32)
    q = np.ascontiguousarray(queries, dtype=np.uint32).reshape(-1, 6)
    ro = np.ascontiguousarray(route_off, dtype=np.uint32)
    rt = np.ascontiguousarray(routed, dtype=np.uint32)
    if rt.size == 0:
        rt = np.zeros(1, dtype=np.uint32)
    nq = q.shape[0]
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    hashes = np.zeros(max(nq, 1), dtype=np.uint64)
    lib.oracle_cpu_backend(_p32(f), _p32(po), po.size - 1, _p32(ko), _p32(k), _p32(q), nq, _p32(ro), _p32(rt),
                           _p64(counts), _p64(hashes), threads)
    return counts[:nq], hashes[:nq]


def subset_of(f, q):
    a = np.ascontiguousarray(f, dtype=np.uint32)
    b = np.ascontiguousarray(q, dtype=np.uint32)
    return bool(_load().oracle_subset_of(_p32(a), _p32(b)))


def filter_less(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    return bool(_load().oracle_filter_less(_p32(a), _p32(b)))


def partition(filters, max_p):
    """Returns a list of partitions, each a sorted tuple of filter indices."""
    lib = _load()
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    n = f.shape[0]
    order = np.zeros(max(n, 1), dtype=np.uint32)
    cap = 2 * n + 1024
    pb = np.zeros(cap, dtype=np.uint32)
    pe = np.zeros(cap, dtype=np.uint32)
    npart = lib.oracle_partition(_p32(f), n, max_p, _p32(order), _p32(pb), _p32(pe), cap)
    if npart < 0:
        raise RuntimeError("oracle_partition failed")
    return [tuple(sorted(int(x) for x in order[pb[i]:pe[i]])) for i in range(npart)]


def masks_of(filters, parts):
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    out = []
    for p in parts:
        m = np.full(6, 0xFFFFFFFF, dtype=np.uint32)
        for i in p:
            m &= f[i]
        out.append(m)
    return out


# ---------------------------------------------------------------------------
# result digests
# ---------------------------------------------------------------------------
def _fin64(z):
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def digest(offsets, keys):
    """Per-query (count, order-independent multiset hash) arrays."""
    offsets = np.asarray(offsets, dtype=np.uint64)
    keys = np.asarray(keys, dtype=np.uint32)
    nq = offsets.size - 1
    counts = (offsets[1:] - offsets[:-1]).astype(np.uint64)
    with np.errstate(over="ignore"):
        h = _fin64(keys.astype(np.uint64) + GOLDEN)
    sums = np.zeros(nq, dtype=np.uint64)
    if keys.size:
        qid = np.repeat(np.arange(nq), counts.astype(np.int64))
        with np.errstate(over="ignore"):
            np.add.at(sums, qid, h)
    return counts, sums


# ---------------------------------------------------------------------------
# the reference's own binaries (oracle/_ref)
# ---------------------------------------------------------------------------
def have_ref():
    return os.path.exists(REF_MATCHER) and os.path.exists(REF_PARTITION)


def write_partition_fib(path, filters, key_off, keys):
    """partition_fib_entry binary records (fib.hh:46-49, fib.cc:14-21)."""
    f = np.ascontiguousarray(filters, dtype=np.uint32).reshape(-1, 6)
    with open(path, "wb") as out:
        for i in range(f.shape[0]):
            b, e = int(key_off[i]), int(key_off[i + 1])
            out.write(struct.pack("<I", 0))
            out.write(f[i].astype("<u4").tobytes())
            out.write(struct.pack("<I", e - b))
            out.write(np.asarray(keys[b:e], dtype="<u4").tobytes())


def run_ref_matcher(filters, key_off, keys, queries, unique=False):
    """Runs the reference's test_matcher; returns (offsets, keys) in its order
    (filter-file order per query); unique sorts/uniques each query."""
    with tempfile.TemporaryDirectory() as d:
        fp, qp = os.path.join(d, "f.bin"), os.path.join(d, "q.bin")
        write_partition_fib(fp, filters, key_off, keys)
        np.ascontiguousarray(queries, dtype="<u4").tofile(qp)
        out = subprocess.run([REF_MATCHER, "F=" + fp, "Q=" + qp], check=True, capture_output=True, text=True).stdout
    offs = [0]
    ks = []
    for line in out.splitlines():
        if not line.startswith("query="):
            continue
        parts = line.split()
        vals = [int(x) for x in parts[1:]]
        if unique:
            vals = sorted(set(vals))
        ks.extend(vals)
        offs.append(len(ks))
    return np.array(offs, dtype=np.uint64), np.array(ks, dtype=np.uint32)


def run_ref_partition(filters, max_p, threads=1):
    """Runs the reference's partitioner; returns (partition_of, masks, sizes)."""
    f = np.ascontiguousarray(filters, dtype="<u4").reshape(-1, 6)
    out = subprocess.run([REF_PARTITION, str(max_p), str(threads)], input=f.tobytes(), check=True,
                         capture_output=True).stdout.decode()
    part = np.zeros(f.shape[0], dtype=np.uint32)
    masks, sizes = {}, {}
    for line in out.splitlines():
        t = line.split()
        if t[0] == "f":
            part[int(t[1])] = int(t[2])
        elif t[0] == "p":
            pid = int(t[1])
            sizes[pid] = int(t[2])
            masks[pid] = np.array([int(x, 16) for x in t[3:9]], dtype=np.uint32)
    np_ = len(sizes)
    return part, np.stack([masks[i] for i in range(np_)]) if np_ else np.zeros((0, 6), np.uint32), \
        np.array([sizes[i] for i in range(np_)], dtype=np.uint32)


def partition_sets(partition_of, n_partitions):
    """Partition membership as a set of frozensets (ids ignored)."""
    groups = [[] for _ in range(n_partitions)]
    for i, p in enumerate(partition_of):
        groups[int(p)].append(i)
    return sorted(tuple(g) for g in groups)
