"""ctypes binding of the C ABI declared in include/tagmatch_b200.h.

The shared library is built in-tree by tagmatch_b200.build.  Loading fails
loudly when it is missing: there is no fallback implementation.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtagmatch_b200.so")
WORKLOAD_PATH = os.path.join(HERE, "libtm_workload.so")

TM_OK = 0
TM_ERR_INVALID = -1
TM_ERR_CUDA = -2
TM_ERR_STATE = -3
TM_ERR_CAPACITY = -4
TM_ERR_NOMEM = -5
TM_ERR_IO = -6
TM_ERR_TIMEOUT = -7
TM_ERR_INTERNAL = -8

STATUS_NAMES = {
    TM_OK: "TM_OK", TM_ERR_INVALID: "TM_ERR_INVALID", TM_ERR_CUDA: "TM_ERR_CUDA", TM_ERR_STATE: "TM_ERR_STATE",
    TM_ERR_CAPACITY: "TM_ERR_CAPACITY", TM_ERR_NOMEM: "TM_ERR_NOMEM", TM_ERR_IO: "TM_ERR_IO",
    TM_ERR_TIMEOUT: "TM_ERR_TIMEOUT", TM_ERR_INTERNAL: "TM_ERR_INTERNAL",
}

u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)
MATCH_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64, u32p, ctypes.c_uint64)
REQUEST_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64, u64p, u32p, ctypes.c_uint32, ctypes.c_int)
TM_FLUSH_FULL_OR_LATENCY = 0
TM_FLUSH_IMMEDIATE = 1
TM_FLUSH_SINGLE = 2
TM_FLUSH_LEARNED = 3
TM_RESULTS_HOST = 0
TM_RESULTS_DEVICE = 1


class TableInfo(ctypes.Structure):
    _fields_ = [("filters", ctypes.c_uint64), ("keys", ctypes.c_uint64), ("partitions", ctypes.c_uint64),
                ("tiles", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64), ("max_key", ctypes.c_uint32)]


class MatchStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint64), ("queries", ctypes.c_uint64), ("routed", ctypes.c_uint64),
                ("items", ctypes.c_uint64), ("pairs", ctypes.c_uint64), ("keys", ctypes.c_uint64),
                ("pair_retries", ctypes.c_uint64), ("match_kernel_launches", ctypes.c_uint64),
                ("match_kernel_ms", ctypes.c_double), ("dense_tests", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("h2d_bytes", ctypes.c_uint64),
                ("d2h_bytes", ctypes.c_uint64), ("records", ctypes.c_uint64)]


class SchedReport(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("steps", ctypes.c_uint64), ("train_mse", ctypes.c_double),
                ("val_mse", ctypes.c_double), ("val_r2", ctypes.c_double), ("mean_mse", ctypes.c_double),
                ("ms", ctypes.c_double)]


f32p = ctypes.POINTER(ctypes.c_float)

# name -> (restype, argtypes); every symbol include/tagmatch_b200.h declares
SIGNATURES = {
    "tm_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p)]),
    "tm_destroy": (None, [ctypes.c_void_p]),
    "tm_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "tm_version": (ctypes.c_char_p, []),
    "tm_add": (ctypes.c_int, [ctypes.c_void_p, u32p, u32p, ctypes.c_uint32]),
    "tm_add_many": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_uint64, u32p, u32p]),
    "tm_remove": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_uint32]),
    "tm_set_database_filename": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "tm_get_database_filename": (ctypes.c_char_p, [ctypes.c_void_p]),
    "tm_set_persistence": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tm_consolidate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    "tm_consolidate_default": (ctypes.c_int, [ctypes.c_void_p]),
    "tm_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    "tm_stop": (ctypes.c_int, [ctypes.c_void_p]),
    "tm_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "tm_set_latency_limit_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "tm_get_latency_limit_ms": (ctypes.c_uint32, [ctypes.c_void_p]),
    "tm_set_batch_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "tm_match_batch": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_uint64, ctypes.c_int, u64p, u32p,
                                      ctypes.c_uint64, u64p]),
    "tm_match_batch_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), u64p,
                                             ctypes.c_void_p]),
    "tm_match_batch_device_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, u64p,
                                                     ctypes.c_void_p]),
    "tm_match_async": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_int, ctypes.c_uint64, MATCH_CALLBACK,
                                      ctypes.c_void_p]),
    "tm_submit": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64, REQUEST_CALLBACK,
                                 ctypes.c_void_p]),
    "tm_set_flush_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tm_set_serving_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tm_set_memory_budget": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "tm_balanced_partitioning": (ctypes.c_int, [u32p, ctypes.c_uint64, ctypes.c_uint32, u32p, u32p, u32p,
                                                ctypes.c_uint64, u64p]),
    "tm_autotune": (ctypes.c_int, [ctypes.c_void_p, u32p, ctypes.c_uint32, u32p, u32p, ctypes.POINTER(ctypes.c_double)]),
    "tm_sched_record": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tm_sched_samples": (ctypes.c_int, [ctypes.c_void_p, f32p, f32p, ctypes.c_uint64, u64p]),
    "tm_sched_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(SchedReport)]),
    "tm_sched_use_order": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tm_sched_predict_batch_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]),
    "tm_set_latency_target_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "tm_mlp_param_count": (ctypes.c_uint32, []),
    "tm_mlp_loss_grad": (ctypes.c_int, [f32p, f32p, f32p, ctypes.c_uint32, f32p, f32p, f32p]),
    "tm_set_tiles_per_item": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "tm_get_tiles_per_item": (ctypes.c_uint32, [ctypes.c_void_p]),
    "tm_get_table_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TableInfo)]),
    "tm_get_match_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(MatchStats)]),
    "tm_reset_match_stats": (ctypes.c_int, [ctypes.c_void_p]),
    "tm_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
}

_lib = None


def load():
    """Loads libtagmatch_b200.so (raises OSError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: run `python -m tagmatch_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TagMatchError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
