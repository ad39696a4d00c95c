"""tcr_search_noalloc: the search for callers that cannot allocate device memory.

Such callers (a host application that hands out a fixed device arena at start-up and forbids
cudaMalloc afterwards, or a plugin host whose allocator the search cannot reach) get one entry
point whose structure and scratch live in a static device array inside the library; they pass
only inputs and outputs.  These tests call it through the C ABI, twice in a row with different
sizes so the second call meets the first call's leftovers in the shared array, and compare every
output with the regular caller-allocated entry points (integer outputs: exact equality).

This file is named to be collected last, so a failure here comes after every other test ran.
"""
import ctypes

import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _desc(x, hx, dmin, dmax, per, mode, L=4096):
    from torchcompactradius_b200 import _lib
    d = _lib.SearchDesc()
    d.dim = x.shape[1]
    d.mode = _lib.MODES[mode]
    d.periodic_mask = sum(1 << k for k, p in enumerate(per) if p)
    d.self_search = 1
    for k in range(x.shape[1]):
        d.domain_min[k] = float(dmin[k])
        d.domain_max[k] = float(dmax[k])
    d.hash_map_length = L
    d.n_query = d.n_ref = x.shape[0]
    d.query_pos = d.ref_pos = x.data_ptr()
    d.query_sup = d.ref_sup = hx.data_ptr()
    return d


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _regular(d, fmt):
    """The caller-allocated path: tcr_build_structure + tcr_count + tcr_emit."""
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    s, w = _lib.search_sizes(d.n_query, d.n_ref, d.dim)
    st = torch.empty(s, dtype=torch.uint8, device="cuda")
    sc = torch.empty(w, dtype=torch.uint8, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.tcr_build_structure(ctypes.byref(d), _vp(st), s, _vp(sc), w, stream), "build")
    off = torch.empty(d.n_query + 1, dtype=torch.int64, device="cuda")
    ip = torch.empty(d.n_query + 1, dtype=torch.int32, device="cuda")
    re = torch.empty(d.n_query, dtype=torch.int64, device="cuda")
    info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
    _lib.check(lib.tcr_count(ctypes.byref(d), _vp(st), _vp(sc), w, None, 0, _vp(off), _vp(ip), _vp(re),
                             ctypes.c_void_p(info.data_ptr()), stream), "count")
    torch.cuda.current_stream().synchronize()
    n = int(info[0])
    col = torch.empty(n, dtype=torch.int64, device="cuda")
    row = torch.empty(n, dtype=torch.int64, device="cuda") if fmt == "coo" else None
    _lib.check(lib.tcr_emit(ctypes.byref(d), _vp(st), _vp(sc), w, None, _vp(off), _vp(row), _vp(col), n, stream),
               "emit")
    torch.cuda.synchronize()
    return off, ip, re, row, col


def _noalloc(d, fmt, capacity):
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    off = torch.full((d.n_query + 1,), -7, dtype=torch.int64, device="cuda")
    ip = torch.full((d.n_query + 1,), -7, dtype=torch.int32, device="cuda")
    re = torch.full((d.n_query,), -7, dtype=torch.int64, device="cuda")
    col = torch.full((capacity,), -7, dtype=torch.int64, device="cuda")
    row = torch.full((capacity,), -7, dtype=torch.int64, device="cuda") if fmt == "coo" else None
    total = ctypes.c_int64(-1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.tcr_search_noalloc(ctypes.byref(d), _vp(off), _vp(ip), _vp(re), _vp(row), _vp(col), capacity,
                                ctypes.byref(total), stream)
    torch.cuda.synchronize()
    return rc, total.value, off, ip, re, row, col


def _case(seed, dim, n, per, hscale):
    x, hx, _, _, dmin, dmax, p = cases.random_case(seed=seed, dim=dim, n=n, nref=None, hscale=hscale,
                                                   extent=[2.0] * dim, periodic=per)
    return torch.tensor(x, device="cuda"), torch.tensor(hx, device="cuda"), dmin, dmax, p


def _check_same(d, fmt):
    off0, ip0, re0, row0, col0 = _regular(d, fmt)
    n = col0.numel()
    rc, total, off1, ip1, re1, row1, col1 = _noalloc(d, fmt, n + 5)
    from torchcompactradius_b200 import _lib
    assert rc == 0, _lib.load().tcr_last_error()
    assert total == n
    assert torch.equal(off0, off1) and torch.equal(ip0, ip1) and torch.equal(re0, re1)
    assert torch.equal(col0, col1[:n]) and bool((col1[n:] == -7).all())
    if fmt == "coo":
        assert torch.equal(row0, row1[:n])
    return n


def test_noalloc_matches_caller_allocated_search_two_calls_in_a_row():
    x1, h1, lo1, hi1, p1 = _case(31, 3, 60000, [True, False, True], 0.09)
    d1 = _desc(x1, h1, lo1, hi1, p1, "symmetric")
    x2, h2, lo2, hi2, p2 = _case(32, 2, 20000, [False, False], 0.03)
    d2 = _desc(x2, h2, lo2, hi2, p2, "gather")
    n1 = _check_same(d1, "coo")
    n2 = _check_same(d2, "csr")   # second call: the array still holds the first call's data
    assert n1 > 0 and n2 > 0
    assert _check_same(d1, "csr") == n1


def test_noalloc_reports_a_too_small_output_without_writing():
    x, h, lo, hi, p = _case(33, 3, 30000, [False] * 3, 0.08)
    d = _desc(x, h, lo, hi, p, "superSymmetric")
    _, _, _, _, col0 = _regular(d, "csr")
    rc, total, _, _, _, _, col = _noalloc(d, "csr", 10)
    assert rc == -1 and total == col0.numel()
    assert bool((col == -7).all())


def test_noalloc_rejects_clouds_beyond_its_static_scratch():
    x = torch.zeros(400000, 3, device="cuda")
    h = torch.full((400000,), 0.01, device="cuda")
    d = _desc(x, h, [0, 0, 0], [1, 1, 1], [False] * 3, "gather")
    rc, total, *_ = _noalloc(d, "csr", 1)
    from torchcompactradius_b200 import _lib
    assert rc == -1 and total == -1
    assert b"static" in _lib.load().tcr_last_error()


def test_noalloc_with_no_queries_writes_no_pairs():
    from torchcompactradius_b200 import _lib
    x, h, lo, hi, p = _case(34, 3, 5000, [False] * 3, 0.08)
    d = _desc(x, h, lo, hi, p, "gather")
    d.self_search = 0
    d.n_query = 0
    d.query_pos = d.query_sup = None
    rc, total, off, ip, re, row, col = _noalloc(d, "coo", 4)
    assert rc == 0, _lib.load().tcr_last_error()
    assert total == 0
    assert int(off[0]) == 0 and int(ip[0]) == 0
    assert bool((col == -7).all()) and bool((row == -7).all())


def test_noalloc_without_a_valid_grid_reports_it_and_writes_no_pairs():
    from torchcompactradius_b200 import _lib
    x = torch.rand(2000, 2, device="cuda")
    h = torch.full((2000,), 1.5, device="cuda")  # support above the periodic extent: no cell grid
    d = _desc(x, h, [0.0, 0.0], [1.0, 1.0], [True, True], "gather")
    rc, total, _, _, _, _, col = _noalloc(d, "csr", 8)
    assert rc == -1 and b"no valid cell grid" in _lib.load().tcr_last_error()
    assert total == 0
    assert bool((col == -7).all())
