"""tm_match_batch_device_noalloc: the matcher for callers that cannot call
cudaMalloc while matching (their device memory belongs to a pool allocator,
or an allocation's device synchronisation is too costly on their serving
path).  It takes all scratch from one static device array; its results must
equal those of tm_match_batch_device, the entry point that allocates, on two
calls in a row (the array keeps the previous call's contents, so the second
call shows that what must start at zero is cleared).

Collected last (file name) so that a failure here comes after every other
test has run; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from tagmatch_b200 import TagMatch, _native, workload
from tests.helpers import wide_key_lists

pytestmark = pytest.mark.gpu


def _cudart():
    for name in ("libcudart.so", "libcudart.so.12"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    import glob
    import os
    for path in glob.glob("/usr/local/cuda*/lib64/libcudart.so*"):
        return ctypes.CDLL(path)
    raise OSError("libcudart not found")


def _d2h(rt, ptr, n, dtype):
    out = np.empty(n, dtype=dtype)
    if n:
        assert rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr), ctypes.c_size_t(out.nbytes), 2) == 0
    return out


def _sorted_per_query(off, keys):
    return [np.sort(keys[int(off[i]):int(off[i + 1])]) for i in range(off.size - 1)]


def _engine(f, ko, k, max_p):
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(f, ko, k)
    tm.consolidate(max_p, 1)
    return tm


def _allocating(lib, rt, tm, dq, n, unique):
    """Results of the existing entry point (which allocates its scratch)."""
    po, pk = ctypes.c_void_p(), ctypes.c_void_p()
    nk = ctypes.c_uint64(0)
    st = lib.tm_match_batch_device(tm._h, ctypes.c_void_p(dq.data_ptr()), n, int(unique), ctypes.byref(po),
                                   ctypes.byref(pk), ctypes.byref(nk), None)
    assert st == 0, lib.tm_last_error(tm._h)
    return _d2h(rt, po.value, n + 1, np.uint64), _d2h(rt, pk.value, nk.value, np.uint32)


def _noalloc(lib, tm, dq, n, unique, d_off, d_keys, capacity=None):
    import torch
    d_off.fill_(-1)
    d_keys.fill_(-1)
    torch.cuda.synchronize()
    got = ctypes.c_uint64(0)
    st = lib.tm_match_batch_device_noalloc(tm._h, ctypes.c_void_p(dq.data_ptr()), n, int(unique),
                                           ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_keys.data_ptr()),
                                           d_keys.numel() if capacity is None else capacity, ctypes.byref(got), None)
    return st, got.value, d_off.cpu().numpy().view(np.uint64)[: n + 1], d_keys.cpu().numpy().view(np.uint32)


def _same(unique, off, keys, ref_off, ref_keys):
    assert np.array_equal(off, ref_off)
    if unique:
        assert np.array_equal(keys, ref_keys)
    else:
        for a, b in zip(_sorted_per_query(off, keys), _sorted_per_query(ref_off, ref_keys)):
            assert np.array_equal(a, b)


# (filters, seed, max partition size, queries, keys): the first case has
# few partitions; the second more than one scan block (2,048) of
# partitions; the third a batch of 4,096 queries (two scan blocks of
# per-query counts) and keys above the 48 KB bitmap of match_unique, so
# that it takes the sort path; the fourth filters with 8..40 keys beside
# filters with 1..7 (the slot-offset path of the key counts and gather).
CASES = [(200_000, 51, 65536, 1500, "plain"), (200_000, 52, 128, 512, "plain"), (200_000, 53, 65536, 4096, "big"),
         (50_000, 54, 65536, 1024, "wide")]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("unique", [False, True])
def test_noalloc_matches_allocating_entry_point(case, unique):
    import torch
    torch.cuda.init()
    rt = _cudart()
    lib = _native.load()
    nf, seed, max_p, n, key_kind = CASES[case]
    f, ko, k = workload.generate_filters(nf, seed)
    big_keys = key_kind == "big"
    if big_keys:
        k = (k.astype(np.uint64) * 977 + 400_000).astype(np.uint32)
    elif key_kind == "wide":
        ko, k = wide_key_lists(nf, seed)
    q = workload.generate_queries(n, f, seed)
    tm = _engine(f, ko, k, max_p)
    info = tm.table_info()
    if case == 1:
        assert 2048 < info["partitions"] <= 16384
    if big_keys:
        assert info["max_key"] >= 48 * 1024 * 8
    dq = torch.from_numpy(q.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ref_off, ref_keys = _allocating(lib, rt, tm, dq, n, unique)
    assert ref_keys.size > 0

    # new entry point, twice in a row, caller-owned outputs
    d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_keys = torch.zeros(ref_keys.size + 16, dtype=torch.int32, device="cuda")
    for _ in range(2):
        st, got, off, keys = _noalloc(lib, tm, dq, n, unique, d_off, d_keys)
        assert st == 0, lib.tm_last_error(tm._h)
        assert got == ref_keys.size
        _same(unique, off, keys[:got], ref_off, ref_keys)

    # an output buffer one key too small: TM_ERR_CAPACITY, the needed count,
    # complete offsets; then a full-size call still gives the same results
    st, got, off, _ = _noalloc(lib, tm, dq, n, unique, d_off, d_keys, capacity=ref_keys.size - 1)
    assert st == _native.TM_ERR_CAPACITY and got == ref_keys.size
    assert np.array_equal(off, ref_off)
    st, got, off, keys = _noalloc(lib, tm, dq, n, unique, d_off, d_keys)
    assert st == 0 and got == ref_keys.size
    _same(unique, off, keys[:got], ref_off, ref_keys)
    tm.close()


def test_noalloc_limits_rejected():
    """Sizes beyond the limits are rejected with a clear error before any
    work: too many queries (TM_ERR_INVALID), and scratch that the array
    cannot hold (TM_ERR_CAPACITY, here the partition queues of 4,096 queries
    routed to ~1,100 of ~5,900 small partitions each)."""
    import torch
    torch.cuda.init()
    lib = _native.load()
    f, ko, k = workload.generate_filters(200_000, 54)
    q = workload.generate_queries(4096, f, 54)
    tm = _engine(f, ko, k, 64)
    d_off = torch.zeros(4098, dtype=torch.int64, device="cuda")
    d_keys = torch.zeros(1 << 20, dtype=torch.int32, device="cuda")
    big = torch.zeros((4097, 6), dtype=torch.int32, device="cuda")
    st, _, _, _ = _noalloc(lib, tm, big, 4097, False, d_off, d_keys)
    assert st == _native.TM_ERR_INVALID and b"at most 4096" in lib.tm_last_error(tm._h)
    dq = torch.from_numpy(q.view(np.int32)).cuda()
    st, _, _, _ = _noalloc(lib, tm, dq, 4096, False, d_off, d_keys)
    assert st == _native.TM_ERR_CAPACITY and b"split the batch" in lib.tm_last_error(tm._h)
    # the engine and the array stay usable: a smaller batch matches
    rt = _cudart()
    ref_off, ref_keys = _allocating(lib, rt, tm, dq, 256, False)
    st, got, off, keys = _noalloc(lib, tm, dq, 256, False, d_off, d_keys)
    assert st == 0 and got == ref_keys.size
    _same(False, off, keys[:got], ref_off, ref_keys)
    tm.close()
