"""ctypes binding of the in-tree C-ABI library ``libtcr_b200.so`` (declared in include/tcr_b200.h).

The product path has no CPU fallback: if the library is missing or no CUDA device is present,
every search raises.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtcr_b200.so")

TCR_OK = 0
MODES = {"gather": 0, "scatter": 1, "symmetric": 2, "superSymmetric": 3}

_lock = threading.Lock()
_lib = None


class SearchDesc(ctypes.Structure):
    """tcr_search_desc (include/tcr_b200.h)."""
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("periodic_mask", ctypes.c_int32),
        ("self_search", ctypes.c_int32),
        ("domain_min", ctypes.c_float * 3),
        ("domain_max", ctypes.c_float * 3),
        ("hash_map_length", ctypes.c_int64),
        ("n_query", ctypes.c_int64),
        ("n_ref", ctypes.c_int64),
        ("query_pos", ctypes.c_void_p),
        ("query_sup", ctypes.c_void_p),
        ("ref_pos", ctypes.c_void_p),
        ("ref_sup", ctypes.c_void_p),
        ("query_ids", ctypes.c_void_p),
        ("ref_ids", ctypes.c_void_p),
        ("hcell", ctypes.c_float * 3),
        ("clamped_grid", ctypes.c_int32),
        ("unit_queries", ctypes.c_int32),
        ("walk_blocks_per_sm", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class CloudDesc(ctypes.Structure):
    """tcr_cloud_desc (include/tcr_b200.h): one cloud of a batch."""
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("periodic_mask", ctypes.c_int32),
        ("domain_min", ctypes.c_float * 3),
        ("domain_max", ctypes.c_float * 3),
        ("hash_map_length", ctypes.c_int64),
        ("n_query", ctypes.c_int64),
        ("n_ref", ctypes.c_int64),
        ("query_pos", ctypes.c_void_p),
        ("query_sup", ctypes.c_void_p),
        ("ref_pos", ctypes.c_void_p),
        ("ref_sup", ctypes.c_void_p),
        ("hcell", ctypes.c_float * 3),
        ("clamped_grid", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class BatchDesc(ctypes.Structure):
    """tcr_batch_desc (include/tcr_b200.h): a batch of independent clouds."""
    _fields_ = [
        ("n_clouds", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("self_search", ctypes.c_int32),
        ("local_index", ctypes.c_int32),
        ("clouds", ctypes.POINTER(CloudDesc)),
        ("query_ids", ctypes.c_void_p),
        ("ref_ids", ctypes.c_void_p),
        ("ref_lin_hint", ctypes.c_void_p),
        ("ref_lin_out", ctypes.c_void_p),
        ("ref_order_out", ctypes.c_void_p),
        ("unit_queries", ctypes.c_int32),
        ("walk_blocks_per_sm", ctypes.c_int32),
    ]


class F64Inputs(ctypes.Structure):
    """tcr_f64_inputs (include/tcr_b200.h): the double arrays of a float64 search."""
    _fields_ = [
        ("query_pos", ctypes.c_void_p),
        ("query_sup", ctypes.c_void_p),
        ("ref_pos", ctypes.c_void_p),
        ("ref_sup", ctypes.c_void_p),
        ("ref_sorted", ctypes.c_void_p),
        ("domain_min", ctypes.c_double * 3),
        ("domain_max", ctypes.c_double * 3),
    ]


class ScatterDesc(ctypes.Structure):
    """tcr_scatter_desc (include/tcr_b200.h): one reduction of values onto an index."""
    _fields_ = [
        ("reduce", ctypes.c_int32),
        ("dtype", ctypes.c_int32),
        ("index_full", ctypes.c_int32),
        ("index_sorted", ctypes.c_int32),
        ("accumulate", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("B", ctypes.c_int64),
        ("E", ctypes.c_int64),
        ("K", ctypes.c_int64),
        ("N", ctypes.c_int64),
        ("src", ctypes.c_void_p),
        ("index", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("arg_out", ctypes.c_void_p),
    ]


REDUCE = {"sum": 0, "mean": 1, "mul": 2, "min": 3, "max": 4}

# name -> (restype, argtypes); every function declared in include/tcr_b200.h
_vp, _i64, _i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
_desc_p = ctypes.POINTER(SearchDesc)
_batch_p = ctypes.POINTER(BatchDesc)
_scatter_p = ctypes.POINTER(ScatterDesc)
SIGNATURES = {
    "tcr_last_error": (ctypes.c_char_p, []),
    "tcr_version": (ctypes.c_int, []),
    "tcr_desc_bytes": (_i64, []),
    "tcr_cloud_desc_bytes": (_i64, []),
    "tcr_batch_desc_bytes": (_i64, []),
    "tcr_kernel_launches": (_i64, []),
    "tcr_profile_kernels": (ctypes.c_int, [_i32]),
    "tcr_profile_kernel_ms": (ctypes.c_int, [_i32, ctypes.POINTER(ctypes.c_float)]),
    "tcr_search_sizes": (ctypes.c_int, [_i64, _i64, _i32, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "tcr_structure_offsets": (ctypes.c_int, [_i64, ctypes.POINTER(_i64), _i32]),
    "tcr_build_structure": (ctypes.c_int, [_desc_p, _vp, _i64, _vp, _i64, _vp]),
    "tcr_count": (ctypes.c_int, [_desc_p, _vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "tcr_emit": (ctypes.c_int, [_desc_p, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp]),
    "tcr_batch_sizes": (ctypes.c_int, [_batch_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "tcr_batch_build_structure": (ctypes.c_int, [_batch_p, _vp, _i64, _vp, _i64, _vp]),
    "tcr_batch_count": (ctypes.c_int, [_batch_p, _vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "tcr_batch_emit": (ctypes.c_int, [_batch_p, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp]),
    "tcr_search_noalloc": (ctypes.c_int, [_desc_p, _vp, _vp, _vp, _vp, _vp, _i64, ctypes.POINTER(_i64), _vp]),
    "tcr_count_f64": (ctypes.c_int, [_desc_p, ctypes.POINTER(F64Inputs), _vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp,
                                     _vp, _vp]),
    "tcr_emit_f64": (ctypes.c_int, [_desc_p, ctypes.POINTER(F64Inputs), _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64,
                                    _vp]),
    "tcr_scatter_desc_bytes": (_i64, []),
    "tcr_index_stats": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp]),
    "tcr_scatter_sizes": (ctypes.c_int, [_scatter_p, ctypes.POINTER(_i64)]),
    "tcr_scatter": (ctypes.c_int, [_scatter_p, _vp, _i64, _vp, _vp]),
}


class TcrError(RuntimeError):
    pass


def load():
    """Loads the library (once) and declares every exported function."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise TcrError(f"{LIB_PATH} is missing: build it with torchcompactradius_b200.build.build() "
                               "(there is no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc, what):
    if rc != TCR_OK:
        msg = load().tcr_last_error()
        raise TcrError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


STRUCT_FIELDS = ["grid", "num_cells", "sorted_points", "sort_index", "cell_start", "cell_lin", "cell_coords",
                 "cell_bucket", "map", "map_capacity"]


def structure_offsets(n_ref):
    arr = (_i64 * len(STRUCT_FIELDS))()
    check(load().tcr_structure_offsets(n_ref, arr, len(STRUCT_FIELDS)), "tcr_structure_offsets")
    return dict(zip(STRUCT_FIELDS, list(arr)))


def search_sizes(n_query, n_ref, dim):
    s, w = _i64(0), _i64(0)
    check(load().tcr_search_sizes(n_query, n_ref, dim, ctypes.byref(s), ctypes.byref(w)), "tcr_search_sizes")
    return s.value, w.value


def scatter_sizes(sdesc):
    w = _i64(0)
    check(load().tcr_scatter_sizes(ctypes.byref(sdesc), ctypes.byref(w)), "tcr_scatter_sizes")
    return w.value


def batch_sizes(bdesc):
    s, w = _i64(0), _i64(0)
    check(load().tcr_batch_sizes(ctypes.byref(bdesc), ctypes.byref(s), ctypes.byref(w)), "tcr_batch_sizes")
    return s.value, w.value


PROFILE_COUNT_WALK = 0
PROFILE_EXPAND = 1


def profile_kernel_ms(kernel):
    ms = ctypes.c_float(0.0)
    check(load().tcr_profile_kernel_ms(kernel, ctypes.byref(ms)), "tcr_profile_kernel_ms")
    return float(ms.value)
