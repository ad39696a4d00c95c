"""ctypes binding of ``liboracle_compact.so`` (the C restatement in ``compact_oracle.c``).

Test infrastructure only; see the header of ``compact_oracle.c`` for the reference lines each
step follows.  ``ensure_built()`` compiles the library with ``make`` when it is missing.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_compact.so")
MODES = {"gather": 0, "scatter": 1, "symmetric": 2, "superSymmetric": 3}
_lib = None


def ensure_built():
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "compact_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        ensure_built()
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, f32p = ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p
        L.oracle_radius_search.restype = vp
        L.oracle_radius_search.argtypes = [ctypes.c_int, i64, f32p, f32p, i64, f32p, f32p, f32p, f32p, vp,
                                           ctypes.c_int, i64]
        L.oracle_brute_force.restype = vp
        L.oracle_brute_force.argtypes = [ctypes.c_int, i64, f32p, f32p, i64, f32p, f32p, f32p, f32p, vp,
                                         ctypes.c_int]
        L.oracle_result_status.argtypes = [vp]
        L.oracle_result_npairs.argtypes = [vp]
        L.oracle_result_npairs.restype = i64
        L.oracle_result_hcell.argtypes = [vp]
        L.oracle_result_hcell.restype = ctypes.c_float
        L.oracle_result_cell_count.argtypes = [vp, vp]
        L.oracle_result_copy.argtypes = [vp, vp, vp]
        L.oracle_result_free.argtypes = [vp]
        L.oracle_wrap.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.oracle_wrap.restype = ctypes.c_float
        L.oracle_compute_hcell.argtypes = [ctypes.c_int, vp, vp, ctypes.c_float, vp]
        L.oracle_compute_hcell.restype = ctypes.c_float
        L.oracle_hash.argtypes = [ctypes.c_int, vp, ctypes.c_uint32]
        L.oracle_hash.restype = ctypes.c_int32
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _f32(a, shape_last=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data


class OracleResult:
    """counts: int64[nq]; col: int64[P] (rows in query order); offsets: int64[nq+1]."""

    def __init__(self, counts, col, hcell=None, cell_count=None):
        self.counts = counts
        self.col = col
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.row = np.repeat(np.arange(len(counts), dtype=np.int64), counts)
        self.hcell = hcell
        self.cell_count = cell_count


def _run(fn, args, with_grid):
    L = lib()
    r = fn(*args)
    try:
        st = L.oracle_result_status(r)
        if st != 0:
            raise ValueError(f"oracle rejected the input (status {st})")
        n = L.oracle_result_npairs(r)
        nq = args[1]
        counts = np.empty(nq, np.int64)
        col = np.empty(n, np.int64)
        L.oracle_result_copy(r, counts.ctypes.data if nq else None, col.ctypes.data if n else None)
        hc, cc = None, None
        if with_grid:
            hc = float(L.oracle_result_hcell(r))
            cc3 = np.zeros(3, np.int32)
            L.oracle_result_cell_count(r, cc3.ctypes.data)
            cc = cc3[:args[0]].copy()
        return OracleResult(counts, col, hc, cc)
    finally:
        L.oracle_result_free(r)


def _prep(xq, hq, xr, hr, dmin, dmax, periodic):
    xq = _f32(xq)
    dim = xq.shape[1]
    hq = None if hq is None else _f32(hq)
    if xr is None:  # the query cloud doubles as the reference cloud (neighborhood.py:187-188)
        xr, hr = xq, hq
    xr = _f32(xr)
    hr = None if hr is None else _f32(hr)
    dmin = _f32(dmin).reshape(dim)
    dmax = _f32(dmax).reshape(dim)
    per = np.ascontiguousarray(np.asarray(periodic, dtype=np.uint8).reshape(dim))
    return dim, xq, hq, xr, hr, dmin, dmax, per


def radius_search(xq, hq, xr, hr, dmin, dmax, periodic, mode="gather", hash_map_length=4096):
    """radiusSearch(..., algorithm='compact') with an explicit domain, in C."""
    dim, xq, hq, xr, hr, dmin, dmax, per = _prep(xq, hq, xr, hr, dmin, dmax, periodic)
    keep = (xq, hq, xr, hr, dmin, dmax, per)  # noqa: F841 (keep buffers alive)
    args = (dim, xq.shape[0], _ptr(xq), _ptr(hq), xr.shape[0], _ptr(xr), _ptr(hr), _ptr(dmin), _ptr(dmax),
            _ptr(per), MODES[mode], int(hash_map_length))
    return _run(lib().oracle_radius_search, args, True)


def brute_force(xq, hq, xr, hr, dmin, dmax, periodic, mode="gather"):
    """All pairs with the reference's distance test and wraps, no grid."""
    dim, xq, hq, xr, hr, dmin, dmax, per = _prep(xq, hq, xr, hr, dmin, dmax, periodic)
    keep = (xq, hq, xr, hr, dmin, dmax, per)  # noqa: F841
    args = (dim, xq.shape[0], _ptr(xq), _ptr(hq), xr.shape[0], _ptr(xr), _ptr(hr), _ptr(dmin), _ptr(dmax),
            _ptr(per), MODES[mode])
    return _run(lib().oracle_brute_force, args, False)


def compute_hcell(dmin, dmax, hmax):
    dmin = _f32(dmin); dmax = _f32(dmax)
    cc = np.zeros(3, np.int32)
    h = lib().oracle_compute_hcell(len(dmin), dmin.ctypes.data, dmax.ctypes.data, float(np.float32(hmax)),
                                   cc.ctypes.data)
    return float(h), cc[:len(dmin)].copy()


def wrap(x, lo, hi):
    return float(lib().oracle_wrap(float(np.float32(x)), float(np.float32(lo)), float(np.float32(hi))))


def hash_cell(cell, L):
    c = np.ascontiguousarray(np.asarray(cell, np.int32))
    return int(lib().oracle_hash(len(c), c.ctypes.data, int(L)))


def num_threads():
    return int(lib().oracle_num_threads())
