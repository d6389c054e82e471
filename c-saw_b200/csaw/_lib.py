"""ctypes binding of libcsaw_b200.so (the C ABI declared in include/csaw.h).

There is no fallback: if the library is missing or fails to load, every call
raises.  Build it with `make -C c-saw_b200` (or __graft_entry__.build()).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libcsaw_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_CAPACITY, ERR_NOMEM, ERR_DEVICE, PENDING = range(7)
MODE_NEIGHBOR, MODE_WALK, MODE_MDRW = 0, 1, 2
BIAS_UNBIASED, BIAS_DEGREE, BIAS_EDGE_WEIGHT, BIAS_HOOK = 0, 1, 2, 3
SCHED_PLAIN, SCHED_BATCHED, SCHED_LEARNED = 0, 1, 2
GRAPH_DEGREE_BIAS, GRAPH_CDF_CACHE, GRAPH_NO_CDF_CACHE = 1, 2, 4
PARAM_DEDUP = 1
MAX_DEPTH = 64
KERNEL_KINDS = {"expand": 0, "heavy": 1, "walk": 2, "mdrw": 3, "setup": 4, "select": 5, "hub": 6, "pair": 7,
                "walk_thread": 8, "persist": 9, "select_thread": 10}

# Every symbol include/csaw.h declares (tests check the library exports them).
EXPORTS = [
    "csaw_last_error", "csaw_version", "csaw_graph_create", "csaw_graph_destroy",
    "csaw_graph_stats", "csaw_graph_profile", "csaw_graph_kernel_stats", "csaw_make_seeds",
    "csaw_sample", "csaw_sample_host", "csaw_sample_batch", "csaw_sample_noalloc", "csaw_sampler_compat",
    "csaw_graph_set_option", "csaw_stream_graph_create", "csaw_stream_graph_destroy", "csaw_stream_sample",
    "csaw_stream_stats", "csaw_stream_graph_cache", "csaw_stream_graph_set_option", "csaw_sched_info", "csaw_sched_get_records", "csaw_sched_train", "csaw_sched_classes", "csaw_sched_get_model", "csaw_sched_set_model",
    "csaw_mlp_grad_host", "csaw_server_create", "csaw_server_destroy", "csaw_server_submit", "csaw_server_wait",
    "csaw_server_get_stats", "csaw_graph_autotune",
]
OPT_CUDA_GRAPHS = 1
OPT_SCHED_RECORD = 2
OPT_GRID_PCT = 3
OPT_PAIR = 4
OPT_HOST_PARTS = 5
OPT_RETRY_SMEM = 6
OPT_PERSISTENT = 7
OPT_THREAD_SELECT = 8
OPT_INCR_REBUILD = 9
STREAM_OPT_READ_IN_PLACE = 1
MLP_NPARAM, MLP_NORM = 1575, 18


class CsawError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"csaw error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("bias", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("n_samples", ctypes.c_int32),
        ("frontier_size", ctypes.c_int32),
        ("neighbor_size", ctypes.c_int32),
        ("depth", ctypes.c_int32),
        ("fanout", ctypes.c_int32 * MAX_DEPTH),
        ("seed", ctypes.c_uint64),
        ("sample_base", ctypes.c_int64),
        ("flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [("n_slots", ctypes.c_int32), ("max_wait_us", ctypes.c_int32), ("device_budget", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int64) for f in ("submitted", "completed", "failed", "queued", "in_flight", "edges",
                                               "peak_device_bytes", "workspace_bytes")] + \
               [(f, ctypes.c_double) for f in ("p50_ms", "p90_ms", "p99_ms", "max_ms", "mean_ms", "p99_queue_ms",
                                                "p99_launch_ms", "p99_gpu_ms", "first_submit_s", "last_done_s",
                                                "max_worker_call_ms")] + \
               [("worker_calls_over_1ms", ctypes.c_int64)]


class TuneResult(ctypes.Structure):
    _fields_ = [("grid_pct", ctypes.c_int32), ("pair", ctypes.c_int32), ("best_ms", ctypes.c_double),
                ("default_ms", ctypes.c_double), ("candidates", ctypes.c_int32), ("persistent", ctypes.c_int32)]


class Job(ctypes.Structure):
    _fields_ = [
        ("params", ctypes.POINTER(Params)),
        ("seeds", ctypes.c_void_p),
        ("out_src", ctypes.c_void_p),
        ("out_dst", ctypes.c_void_p),
        ("out_sample", ctypes.c_void_p),
        ("out_depth", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("n_out", ctypes.c_int64),
        ("status", ctypes.c_int32),
        ("host_buffers", ctypes.c_int32),
    ]


class StreamInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "n_partitions", "n_slots", "partition_loads", "partition_hits", "bytes_h2d", "kernel_launches",
        "host_pinned_in_place", "items_read_in_place")]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "n_vertices", "n_edges", "max_degree", "device_bytes", "workspace_bytes",
        "kernel_launches", "last_edges", "last_items", "last_bytes")]


_L = None


def lib():
    """Load the library (raises if it is not built)."""
    global _L
    if _L is not None:
        return _L
    if not os.path.exists(LIB_PATH):
        raise CsawError(ERR_CUDA, f"{LIB_PATH} is not built: run `make -C c-saw_b200`")
    L = ctypes.CDLL(LIB_PATH)
    p, i32, i64, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64
    P64 = ctypes.POINTER(ctypes.c_int64)
    L.csaw_last_error.restype = ctypes.c_char_p
    L.csaw_version.restype = ctypes.c_char_p
    L.csaw_graph_create.argtypes = [p, i32, p, p, i64, i64, i32, ctypes.POINTER(p)]
    L.csaw_graph_destroy.argtypes = [p]
    L.csaw_graph_stats.argtypes = [p, ctypes.POINTER(Stats)]
    L.csaw_graph_profile.argtypes = [p, i32]
    L.csaw_graph_kernel_stats.argtypes = [p, i32, ctypes.POINTER(ctypes.c_double), P64, P64, P64]
    L.csaw_make_seeds.argtypes = [p, i64, u64, p, p]
    sig = [p, ctypes.POINTER(Params), p, p, p, p, p, i64, P64, p]
    L.csaw_sample.argtypes = sig
    L.csaw_sample_host.argtypes = sig
    L.csaw_sample_noalloc.argtypes = sig
    L.csaw_sample_batch.argtypes = [p, ctypes.POINTER(Job), i32, p]
    L.csaw_graph_set_option.argtypes = [p, i32, i64]
    L.csaw_stream_graph_create.argtypes = [p, i32, p, p, i64, i64, i32, i64, ctypes.POINTER(p)]
    L.csaw_stream_graph_destroy.argtypes = [p]
    L.csaw_stream_sample.argtypes = sig
    L.csaw_stream_stats.argtypes = [p, ctypes.POINTER(StreamInfo)]
    L.csaw_stream_graph_cache.argtypes = [p, i32]
    L.csaw_stream_graph_set_option.argtypes = [p, i32, ctypes.c_int64]
    PF = ctypes.POINTER(ctypes.c_float)
    L.csaw_sched_info.argtypes = [p, P64, ctypes.POINTER(ctypes.c_int), PF]
    L.csaw_sched_train.argtypes = [p, i32, ctypes.c_float, u64, PF]
    L.csaw_sched_classes.argtypes = [p, ctypes.POINTER(ctypes.c_uint32)]
    L.csaw_sched_get_records.argtypes = [p, p, i64, P64]
    L.csaw_sched_get_model.argtypes = [p, p, p]
    L.csaw_sched_set_model.argtypes = [p, p, p]
    L.csaw_mlp_grad_host.argtypes = [p, p, p, i32, p, PF]
    L.csaw_graph_autotune.argtypes = [p, ctypes.POINTER(Job), i32, p, ctypes.POINTER(TuneResult)]
    L.csaw_server_create.argtypes = [p, ctypes.POINTER(ServerConfig), ctypes.POINTER(p)]
    L.csaw_server_destroy.argtypes = [p]
    L.csaw_server_submit.argtypes = [p, ctypes.POINTER(Params), p, p, p, p, p, i64, ctypes.POINTER(ctypes.c_uint64)]
    L.csaw_server_wait.argtypes = [p, ctypes.c_uint64, i64, P64, ctypes.POINTER(ctypes.c_double)]
    L.csaw_server_get_stats.argtypes = [p, i32, ctypes.POINTER(ServerStats)]
    L.csaw_sampler_compat.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i32, i32, i32, i32, i32, i32,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTS:
        if name not in ("csaw_last_error", "csaw_version"):
            getattr(L, name).restype = ctypes.c_int
    _L = L
    return L


def check(rc):
    if rc != OK:
        raise CsawError(rc, lib().csaw_last_error().decode())
    return rc
