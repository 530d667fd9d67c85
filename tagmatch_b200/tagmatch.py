"""Python mirror of the reference's tagmatch API (tagmatch.hh:11-37).

    tm = TagMatch()
    tm.add(filter, [k1, k2]); tm.consolidate(65536)
    offsets, keys = tm.match_batch(queries)               # tagmatch::match, whole batch
    offsets, keys = tm.match_batch(queries, unique=True)  # tagmatch::match_unique
    tm.start(); tm.match(q, handler); tm.stop()           # asynchronous, handler(tag, keys)

Filters/queries: numpy uint32 [n, 6] (bit p = bit p % 32 of word p / 32), or
the reference's 192-character '0'/'1' strings (character i = bit i).
"""
import ctypes
import threading

import numpy as np

from . import _native
from ._native import TagMatchError, load, u32p, u64p

FILTER_WORDS = 6


def filter_from_string(s):
    """The reference's string constructor (bitvector.hh:112-128): char i = bit i."""
    w = np.zeros(FILTER_WORDS, dtype=np.uint32)
    for i, c in enumerate(s[:192]):
        if c == "1":
            w[i >> 5] |= np.uint32(1 << (i & 31))
    return w


def filter_to_string(w):
    w = np.asarray(w, dtype=np.uint32)
    return "".join("1" if (int(w[p >> 5]) >> (p & 31)) & 1 else "0" for p in range(192))


def filter_from_bits(bits):
    w = np.zeros(FILTER_WORDS, dtype=np.uint32)
    for p in bits:
        w[p >> 5] |= np.uint32(1 << (p & 31))
    return w


def as_filter(f):
    if isinstance(f, str):
        return filter_from_string(f)
    a = np.ascontiguousarray(f, dtype=np.uint32).reshape(-1)
    if a.size != FILTER_WORDS:
        raise ValueError("a filter is 6 uint32 words")
    return a


def as_filters(fs):
    if isinstance(fs, (list, tuple)) and fs and isinstance(fs[0], str):
        return np.stack([filter_from_string(s) for s in fs])
    a = np.ascontiguousarray(fs, dtype=np.uint32)
    if a.size == 0:
        return a.reshape(0, FILTER_WORDS)
    return a.reshape(-1, FILTER_WORDS)


def _p32(a):
    return a.ctypes.data_as(u32p)


def _p64(a):
    return a.ctypes.data_as(u64p)


class TagMatch:
    """One engine; the reference's static class methods become methods."""

    def __init__(self):
        self._lib = load()
        h = ctypes.c_void_p()
        self._check(self._lib.tm_create(ctypes.byref(h)), h)
        self._h = h
        self._callbacks = {}
        self._cb_lock = threading.Lock()
        self._next_tag = 1
        self._cfunc = _native.MATCH_CALLBACK(self._on_done)
        self._rfunc = _native.REQUEST_CALLBACK(self._on_request)

    # -- plumbing --------------------------------------------------------
    def _check(self, st, h=None):
        if st != _native.TM_OK:
            msg = self._lib.tm_last_error(h if h is not None else self._h)
            raise TagMatchError(st, (msg or b"").decode(errors="replace"))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- staging (tagmatch.cc:62-77) --------------------------------------
    def add(self, f, keys):
        w = as_filter(f)
        k = np.atleast_1d(np.asarray(keys, dtype=np.uint32))
        self._check(self._lib.tm_add(self._h, _p32(w), _p32(k), k.size))

    def add_many(self, filters, key_offsets, keys):
        f = as_filters(filters)
        ko = np.ascontiguousarray(key_offsets, dtype=np.uint32)
        k = np.ascontiguousarray(keys, dtype=np.uint32)
        if k.size == 0:
            k = np.zeros(1, dtype=np.uint32)
        self._check(self._lib.tm_add_many(self._h, _p32(f), f.shape[0], _p32(ko), _p32(k)))

    def remove(self, f, key):
        w = as_filter(f)
        self._check(self._lib.tm_remove(self._h, _p32(w), int(key)))

    # -- database (tagmatch.cc:79-87) ---------------------------------------
    def set_database_filename(self, name):
        self._check(self._lib.tm_set_database_filename(self._h, str(name).encode()))

    def get_database_filename(self):
        return self._lib.tm_get_database_filename(self._h).decode()

    def set_persistence(self, on):
        self._check(self._lib.tm_set_persistence(self._h, 1 if on else 0))

    # -- lifecycle (tagmatch.cc:92-198) -------------------------------------
    def consolidate(self, partition_size=None, threads=1):
        if partition_size is None:
            self._check(self._lib.tm_consolidate_default(self._h))
        else:
            self._check(self._lib.tm_consolidate(self._h, partition_size, threads))

    def start(self, threads=4, gpu_count=1):
        self._check(self._lib.tm_start(self._h, threads, gpu_count))

    def stop(self):
        self._check(self._lib.tm_stop(self._h))

    def clear(self):
        self._check(self._lib.tm_clear(self._h))

    def set_latency_limit_ms(self, ms):
        self._check(self._lib.tm_set_latency_limit_ms(self._h, ms))

    def get_latency_limit_ms(self):
        return self._lib.tm_get_latency_limit_ms(self._h)

    def set_batch_limit(self, queries):
        self._check(self._lib.tm_set_batch_limit(self._h, queries))

    # -- matching (tagmatch.cc:200-210) -------------------------------------
    def match_batch(self, queries, unique=False, capacity=None):
        """Returns (offsets [n + 1] uint64, keys uint32)."""
        q = as_filters(queries)
        n = q.shape[0]
        off = np.zeros(n + 1, dtype=np.uint64)
        cap = capacity if capacity is not None else max(1024, n * 64)
        for _ in range(3):
            keys = np.empty(max(cap, 1), dtype=np.uint32)
            nk = ctypes.c_uint64(0)
            st = self._lib.tm_match_batch(self._h, _p32(q) if n else None, n, 1 if unique else 0, _p64(off),
                                          _p32(keys), cap, ctypes.byref(nk))
            if st == _native.TM_ERR_CAPACITY:
                cap = int(nk.value)
                continue
            self._check(st)
            return off, keys[: nk.value]
        raise TagMatchError(_native.TM_ERR_CAPACITY, "output capacity did not converge")

    def match(self, query, handler, unique=False):
        """Queues one query; handler(keys: np.ndarray) runs on an engine thread."""
        w = as_filter(query)
        with self._cb_lock:
            tag = self._next_tag
            self._next_tag += 1
            self._callbacks[tag] = handler
        st = self._lib.tm_match_async(self._h, _p32(w), 1 if unique else 0, tag, self._cfunc, None)
        if st != _native.TM_OK:
            with self._cb_lock:
                self._callbacks.pop(tag, None)
            self._check(st)
        return tag

    def submit(self, queries, handler, unique=False):
        """Queues a request of n queries; handler(offsets, keys, status) runs
        once, on an engine thread, with the request's results."""
        q = as_filters(queries)
        with self._cb_lock:
            tag = self._next_tag
            self._next_tag += 1
            self._callbacks[tag] = handler
        st = self._lib.tm_submit(self._h, _p32(q) if q.shape[0] else None, q.shape[0], 1 if unique else 0, tag,
                                 self._rfunc, None)
        if st != _native.TM_OK:
            with self._cb_lock:
                self._callbacks.pop(tag, None)
            self._check(st)
        return tag

    def set_flush_mode(self, mode):
        self._check(self._lib.tm_set_flush_mode(self._h, mode))

    def set_memory_budget(self, nbytes):
        self._check(self._lib.tm_set_memory_budget(self._h, nbytes))

    def set_serving_results(self, where):
        """TM_RESULTS_HOST or TM_RESULTS_DEVICE (request keys left in device
        memory; this wrapper copies them out inside the callback)."""
        self._check(self._lib.tm_set_serving_results(self._h, where))
        self._device_results = where == _native.TM_RESULTS_DEVICE

    def _on_request(self, user, tag, offsets, keys, n, status):
        off = np.ctypeslib.as_array(offsets, shape=(n + 1,)).copy()
        nk = int(off[-1])
        if not nk:
            arr = np.zeros(0, dtype=np.uint32)
        elif getattr(self, "_device_results", False):
            arr = read_device(ctypes.cast(keys, ctypes.c_void_p).value, nk, np.uint32)
        else:
            arr = np.ctypeslib.as_array(keys, shape=(nk,)).copy()
        with self._cb_lock:
            h = self._callbacks.pop(tag, None)
        if h is not None:
            h(off, arr, status)

    def match_unique(self, query, handler):
        return self.match(query, handler, unique=True)

    def _on_done(self, user, tag, keys, n):
        arr = np.ctypeslib.as_array(keys, shape=(n,)).copy() if n else np.zeros(0, dtype=np.uint32)
        with self._cb_lock:
            h = self._callbacks.pop(tag, None)
        if h is not None:
            h(arr)

    # -- introspection ------------------------------------------------------
    def table_info(self):
        info = _native.TableInfo()
        self._check(self._lib.tm_get_table_info(self._h, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in info._fields_}

    def autotune(self, sample_queries):
        """Picks tiles per work item and the device batch size on a sample
        (device timing); returns (seg_tiles, batch_limit, queries_per_s)."""
        q = as_filters(sample_queries)
        seg, bl = ctypes.c_uint32(0), ctypes.c_uint32(0)
        qps = ctypes.c_double(0)
        self._check(self._lib.tm_autotune(self._h, _p32(q), q.shape[0], ctypes.byref(seg), ctypes.byref(bl),
                                          ctypes.byref(qps)))
        return seg.value, bl.value, qps.value

    # -- learned scheduler ---------------------------------------------------
    def sched_record(self, on):
        """Record per-work-item timings of every batch as cost-model samples."""
        self._check(self._lib.tm_sched_record(self._h, 1 if on else 0))

    def sched_samples(self):
        """Returns (features [n, 8] float32, log warp-cycles [n] float32)."""
        n = ctypes.c_uint64(0)
        self._check(self._lib.tm_sched_samples(self._h, None, None, 0, ctypes.byref(n)))
        x = np.zeros((n.value, 8), dtype=np.float32)
        t = np.zeros(n.value, dtype=np.float32)
        f32 = ctypes.POINTER(ctypes.c_float)
        self._check(self._lib.tm_sched_samples(self._h, x.ctypes.data_as(f32), t.ctypes.data_as(f32), n.value,
                                               ctypes.byref(n)))
        return x, t

    def sched_train(self, epochs=20):
        """Trains the cost model on the GPU; returns its report as a dict."""
        rep = _native.SchedReport()
        self._check(self._lib.tm_sched_train(self._h, epochs, ctypes.byref(rep)))
        return {k: getattr(rep, k) for k, _ in rep._fields_}

    def sched_use_order(self, on):
        self._check(self._lib.tm_sched_use_order(self._h, 1 if on else 0))

    def sched_predict_batch_ms(self, queries):
        ms = ctypes.c_double(0)
        self._check(self._lib.tm_sched_predict_batch_ms(self._h, queries, ctypes.byref(ms)))
        return ms.value

    def set_latency_target_ms(self, ms):
        self._check(self._lib.tm_set_latency_target_ms(self._h, ms))

    def set_tiles_per_item(self, seg_tiles):
        """Tiles per work item of the subset test (the autotuner's knob)."""
        self._check(self._lib.tm_set_tiles_per_item(self._h, seg_tiles))

    def get_tiles_per_item(self):
        return self._lib.tm_get_tiles_per_item(self._h)

    def set_profiling(self, on):
        self._check(self._lib.tm_set_profiling(self._h, 1 if on else 0))

    def reset_match_stats(self):
        self._check(self._lib.tm_reset_match_stats(self._h))

    def match_batch_device(self, d_queries_ptr, n, unique=False, stream=0):
        """Device-resident batch: returns (d_offsets_ptr, d_keys_ptr, n_keys)."""
        po, pk = ctypes.c_void_p(), ctypes.c_void_p()
        nk = ctypes.c_uint64(0)
        self._check(self._lib.tm_match_batch_device(self._h, ctypes.c_void_p(d_queries_ptr), n, 1 if unique else 0,
                                                     ctypes.byref(po), ctypes.byref(pk), ctypes.byref(nk),
                                                     ctypes.c_void_p(stream)))
        return po.value, pk.value, nk.value

    def match_stats(self):
        st = _native.MatchStats()
        self._check(self._lib.tm_get_match_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}


_cudart_lib = None


def _cudart():
    global _cudart_lib
    if _cudart_lib is None:
        import glob
        names = ["libcudart.so.12", "libcudart.so"] + sorted(glob.glob("/usr/local/cuda*/lib64/libcudart.so*"))
        for name in names:
            try:
                _cudart_lib = ctypes.CDLL(name)
                break
            except OSError:
                continue
        else:
            raise OSError("libcudart not found")
    return _cudart_lib


def read_device(ptr, count, dtype):
    """Copies count elements of dtype from device address ptr (as returned by
    match_batch_device) into a new numpy array (synchronous cudaMemcpy)."""
    out = np.empty(int(count), dtype=dtype)
    if out.size:
        st = _cudart().cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr), ctypes.c_size_t(out.nbytes),
                                  2)
        if st != 0:
            raise TagMatchError(_native.TM_ERR_CUDA, f"cudaMemcpy device->host failed ({st})")
    return out


def mlp_loss_grad(params, features, targets):
    """The cost model's GPU kernels on given data: (outputs [n], gradient of
    the mean squared error [P], loss)."""
    lib = load()
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 8)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    n = x.shape[0]
    y = np.zeros(max(n, 1), dtype=np.float32)
    g = np.zeros(p.size, dtype=np.float32)
    loss = ctypes.c_float(0)
    f32 = ctypes.POINTER(ctypes.c_float)
    st = lib.tm_mlp_loss_grad(p.ctypes.data_as(f32), x.ctypes.data_as(f32), t.ctypes.data_as(f32), n,
                              y.ctypes.data_as(f32), g.ctypes.data_as(f32), ctypes.byref(loss))
    if st != _native.TM_OK:
        raise TagMatchError(st, "tm_mlp_loss_grad failed")
    return y[:n], g, loss.value


def balanced_partitioning(filters, max_p):
    """partitioning::balanced_partitioning on the GPU (partitioning.cc:361-411).

    Returns (partition_of [n], masks [P, 6], sizes [P]).
    """
    lib = load()
    f = as_filters(filters)
    n = f.shape[0]
    part = np.zeros(max(n, 1), dtype=np.uint32)
    cap = max(16, n // 16 + 64)
    for _ in range(3):
        masks = np.zeros((cap, FILTER_WORDS), dtype=np.uint32)
        sizes = np.zeros(cap, dtype=np.uint32)
        npart = ctypes.c_uint64(0)
        st = lib.tm_balanced_partitioning(_p32(f) if n else None, n, max_p, _p32(part), _p32(masks), _p32(sizes), cap,
                                          ctypes.byref(npart))
        if st == _native.TM_ERR_CAPACITY:
            cap = int(npart.value)
            continue
        if st != _native.TM_OK:
            raise TagMatchError(st, "balanced_partitioning failed")
        p = int(npart.value)
        return part[:n], masks[:p], sizes[:p]
    raise TagMatchError(_native.TM_ERR_CAPACITY, "partition capacity did not converge")
