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


@pytest.mark.parametrize("unique", [False, True])
def test_noalloc_matches_allocating_entry_point(unique):
    import torch
    torch.cuda.init()
    rt = _cudart()
    lib = _native.load()
    f, ko, k = workload.generate_filters(200_000, 51)
    q = workload.generate_queries(1500, f, 51)
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(f, ko, k)
    tm.consolidate(65536, 1)
    dq = torch.from_numpy(q.view(np.int32)).cuda()
    n = q.shape[0]
    torch.cuda.synchronize()

    # existing entry point (allocates its scratch)
    po, pk = ctypes.c_void_p(), ctypes.c_void_p()
    nk = ctypes.c_uint64(0)
    st = lib.tm_match_batch_device(tm._h, ctypes.c_void_p(dq.data_ptr()), n, int(unique), ctypes.byref(po),
                                   ctypes.byref(pk), ctypes.byref(nk), None)
    assert st == 0, lib.tm_last_error(tm._h)
    ref_off = _d2h(rt, po.value, n + 1, np.uint64)
    ref_keys = _d2h(rt, pk.value, nk.value, np.uint32)
    assert ref_keys.size > 0

    # new entry point, twice in a row, caller-owned outputs
    d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_keys = torch.zeros(ref_keys.size + 16, dtype=torch.int32, device="cuda")
    for _ in range(2):
        d_off.fill_(-1)
        d_keys.fill_(-1)
        torch.cuda.synchronize()
        got = ctypes.c_uint64(0)
        st = lib.tm_match_batch_device_noalloc(tm._h, ctypes.c_void_p(dq.data_ptr()), n, int(unique),
                                               ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_keys.data_ptr()),
                                               d_keys.numel(), ctypes.byref(got), None)
        assert st == 0, lib.tm_last_error(tm._h)
        assert got.value == ref_keys.size
        off = d_off.cpu().numpy().view(np.uint64)
        keys = d_keys.cpu().numpy().view(np.uint32)[: got.value]
        assert np.array_equal(off, ref_off)
        if unique:
            assert np.array_equal(keys, ref_keys)
        else:
            for a, b in zip(_sorted_per_query(off, keys), _sorted_per_query(ref_off, ref_keys)):
                assert np.array_equal(a, b)

    # limits are rejected with a clear error, nothing is written
    big = torch.zeros((4097, 6), dtype=torch.int32, device="cuda")
    got = ctypes.c_uint64(0)
    st = lib.tm_match_batch_device_noalloc(tm._h, ctypes.c_void_p(big.data_ptr()), 4097, 0,
                                           ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_keys.data_ptr()),
                                           d_keys.numel(), ctypes.byref(got), None)
    assert st == _native.TM_ERR_INVALID and b"at most 4096" in lib.tm_last_error(tm._h)
    tm.close()
