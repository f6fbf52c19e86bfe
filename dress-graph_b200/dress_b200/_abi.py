"""ctypes binding of libdress_cuda.so (the B200 engine's C ABI).

The structures mirror ``include/dress_b200.h`` (which is ABI-identical to the
reference's ``libdress/include/dress/dress.h:12-75``).  Loading fails loudly
when the library has not been built: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libdress_cuda.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_c_i64_p = ctypes.POINTER(ctypes.c_int64)


class DressGraph(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int), ("N", ctypes.c_int), ("E", ctypes.c_int),
        ("U", _c_int_p), ("V", _c_int_p),
        ("adj_offset", _c_int_p), ("adj_target", _c_int_p), ("adj_edge_idx", _c_int_p),
        ("max_degree", ctypes.c_int),
        ("W", _c_dbl_p), ("edge_weight", _c_dbl_p), ("edge_dress", _c_dbl_p),
        ("edge_dress_next", _c_dbl_p), ("NW", _c_dbl_p), ("vertex_dress", _c_dbl_p),
        ("precompute_intercepts", ctypes.c_int),
        ("intercept_offset", _c_int_p), ("intercept_edge_ux", _c_int_p),
        ("intercept_edge_vx", _c_int_p),
    ]


PGraph = ctypes.POINTER(DressGraph)


class HistPair(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("count", ctypes.c_int64)]


class HistRequest(ctypes.Structure):
    _fields_ = [
        ("graph", PGraph), ("kind", ctypes.c_int), ("k", ctypes.c_int),
        ("max_iterations", ctypes.c_int), ("epsilon", ctypes.c_double),
        ("n_samples", ctypes.c_int), ("seed", ctypes.c_uint),
        ("offset", ctypes.c_int), ("stride", ctypes.c_int),
        ("want_histogram", ctypes.c_int), ("keep_multisets", ctypes.c_int),
        ("hist_flat", _c_i64_p), ("hist_len", ctypes.c_int),
        ("multisets", _c_dbl_p), ("num_subgraphs", ctypes.c_int64),
        ("fits", ctypes.c_int64), ("status", ctypes.c_int),
    ]


class Config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int), ("memory_budget_bytes", ctypes.c_size_t),
        ("fit_chunk", ctypes.c_int), ("group_threads", ctypes.c_int),
        ("exact_sums", ctypes.c_int), ("one_launch_max_edges", ctypes.c_int), ("reserved", ctypes.c_int * 6),
    ]


class FitStats(ctypes.Structure):
    _fields_ = [("common_terms", ctypes.c_int64), ("sweeps", ctypes.c_int),
                ("setup_ms", ctypes.c_double), ("iterate_ms", ctypes.c_double),
                ("vertex_bin_items", ctypes.c_int64 * 8), ("vertex_bin_terms", ctypes.c_int64 * 8),
                ("edge_bin_items", ctypes.c_int64 * 8), ("edge_bin_terms", ctypes.c_int64 * 8),
                ("phase_ms", ctypes.c_double * 5)]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int), ("memory_budget_bytes", ctypes.c_size_t),
        ("lanes", ctypes.c_int), ("launch_slots", ctypes.c_int),
        ("launch_work", ctypes.c_int64), ("finishers", ctypes.c_int),
        ("max_queued", ctypes.c_int), ("reserved", ctypes.c_int * 8),
    ]


class ServerRequest(ctypes.Structure):
    _fields_ = [
        ("graph", PGraph), ("kind", ctypes.c_int), ("k", ctypes.c_int),
        ("max_iterations", ctypes.c_int), ("epsilon", ctypes.c_double),
        ("iterations", ctypes.c_int), ("delta", ctypes.c_double),
        ("hist_flat", _c_i64_p), ("hist_len", ctypes.c_int),
        ("num_subgraphs", ctypes.c_int64), ("fits", ctypes.c_int64),
        ("edge_sweeps", ctypes.c_int64), ("path", ctypes.c_int), ("status", ctypes.c_int),
        ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
        ("reserved_bytes", ctypes.c_int64), ("done", ctypes.c_int),
    ]


class ServerClassStats(ctypes.Structure):
    _fields_ = [
        ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
        ("queue_p50_ms", ctypes.c_double), ("queue_p99_ms", ctypes.c_double),
    ]


SERVER_CLASSES = ("fit_batch", "fit_lane", "hist_batch", "hist_lane")


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("elapsed_s", ctypes.c_double),
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
        ("cancelled", ctypes.c_int64), ("rejected", ctypes.c_int64),
        ("fits", ctypes.c_int64), ("edge_sweeps", ctypes.c_int64), ("batch_launches", ctypes.c_int64),
        ("budget_bytes", ctypes.c_int64), ("reserved_bytes", ctypes.c_int64),
        ("peak_reserved_bytes", ctypes.c_int64), ("pool_bytes", ctypes.c_int64),
        ("max_in_service", ctypes.c_int),
        ("device_busy_ms", ctypes.c_double), ("device_work_ms", ctypes.c_double),
        ("cls", ServerClassStats * 4),
    ]


_HIST_ARGS = [PGraph, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
              ctypes.c_uint, _c_int_p, ctypes.c_int, ctypes.POINTER(_c_dbl_p), _c_i64_p]

# name -> (restype, argtypes); every entry point declared in include/*.h
SIGNATURES = {
    "dress_init_graph": (PGraph, [ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p, _c_dbl_p,
                                  _c_dbl_p, ctypes.c_int, ctypes.c_int]),
    "dress_free_graph": (None, [PGraph]),
    "dress_fit": (None, [PGraph, ctypes.c_int, ctypes.c_double, _c_int_p, _c_dbl_p]),
    "dress_fit_cuda": (None, [PGraph, ctypes.c_int, ctypes.c_double, _c_int_p, _c_dbl_p]),
    "dress_delta_fit_cuda": (ctypes.POINTER(HistPair), _HIST_ARGS),
    "dress_delta_fit_cuda_strided": (ctypes.POINTER(HistPair), _HIST_ARGS + [ctypes.c_int, ctypes.c_int]),
    "dress_delta_fit_cuda_strided_flat": (_c_i64_p, _HIST_ARGS + [ctypes.c_int, ctypes.c_int]),
    "dress_delta_fit_cuda_flat": (_c_i64_p, _HIST_ARGS),
    "dress_nabla_fit_cuda": (ctypes.POINTER(HistPair), _HIST_ARGS),
    "dress_nabla_fit_cuda_strided": (ctypes.POINTER(HistPair), _HIST_ARGS + [ctypes.c_int, ctypes.c_int]),
    "dress_nabla_fit_cuda_flat": (_c_i64_p, _HIST_ARGS),
    "dress_nabla_fit_cuda_strided_flat": (_c_i64_p, _HIST_ARGS + [ctypes.c_int, ctypes.c_int]),
    "dressx_configure": (ctypes.c_int, [ctypes.POINTER(Config)]),
    "dressx_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "dressx_fit": (ctypes.c_int, [PGraph, ctypes.c_int, ctypes.c_double, _c_int_p, _c_dbl_p]),
    "dressx_last_fit_stats": (ctypes.c_int, [ctypes.POINTER(FitStats)]),
    "dressx_hist_batch": (ctypes.c_int, [ctypes.POINTER(HistRequest), ctypes.c_int]),
    "dressx_hist_batch_per_fit": (ctypes.c_int, [ctypes.POINTER(HistRequest), ctypes.c_int]),
    "dressx_free": (None, [ctypes.c_void_p]),
    "dressx_batch_create": (ctypes.c_int, [ctypes.POINTER(HistRequest), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "dressx_batch_run": (ctypes.c_int, [ctypes.c_void_p]),
    "dressx_batch_fetch": (ctypes.c_int, [ctypes.c_void_p]),
    "dressx_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p, ctypes.POINTER(ctypes.c_float)]),
    "dressx_batch_capture": (ctypes.c_int, [ctypes.c_void_p]),
    "dressx_batch_stats": (ctypes.c_int, [ctypes.c_void_p, _c_i64_p, _c_i64_p, _c_i64_p]),
    "dressx_batch_timing": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p]),
    "dressx_batch_destroy": (None, [ctypes.c_void_p]),
    "dressx_stream": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p)]),
    "dressx_counters": (ctypes.c_int, [_c_i64_p, _c_i64_p, _c_i64_p, ctypes.c_int]),
    "dressx_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "dressx_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerRequest)]),
    "dressx_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerRequest), ctypes.c_int]),
    "dressx_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerRequest)]),
    "dressx_server_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dressx_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats), ctypes.c_int]),
    "dressx_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dressx_server_estimate": (ctypes.c_int, [PGraph, ctypes.c_int, ctypes.c_int, _c_i64_p, _c_int_p]),
    "dressx_init_graph": (PGraph, [ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p, _c_dbl_p,
                                   _c_dbl_p, ctypes.c_int, ctypes.c_int]),
    "dressx_get_batch": (ctypes.c_int, [PGraph, _c_int_p, _c_int_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                        _c_dbl_p, ctypes.c_double, _c_dbl_p]),
    "dressx_hist_merge": (ctypes.c_int, [ctypes.POINTER(_c_i64_p), _c_i64_p, ctypes.c_int,
                                         ctypes.POINTER(_c_i64_p), _c_i64_p]),
    "dressx_histogram_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p]),
}

NOALLOC_MAX_VALUES = 1 << 20          # DRESSX_NOALLOC_MAX_VALUES

_lib = None


def load(path=LIB_PATH):
    """Load and bind the engine library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libdress_cuda.so not built at {path}; run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error():
    lib = load()
    buf = ctypes.create_string_buffer(512)
    code = lib.dressx_last_error(buf, 512)
    return code, buf.value.decode(errors="replace")
