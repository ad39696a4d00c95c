"""C-ABI boundary checks that need no GPU: the library loads, exports every declared symbol,
the ctypes descriptor matches the C layout, and the host-side validation rejects bad input."""
import ctypes
import os
import re

import pytest
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(REPO, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(REPO, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(tcr_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    declared = _declared()
    assert {"tcr_build_structure", "tcr_count", "tcr_emit", "tcr_search_sizes"} <= declared
    for name in declared:
        assert hasattr(lib, name), name
    assert declared <= set(_lib.SIGNATURES), declared - set(_lib.SIGNATURES)


def test_descriptor_layout_matches_library():
    from torchcompactradius_b200 import _lib
    assert ctypes.sizeof(_lib.SearchDesc) == _lib.load().tcr_desc_bytes()
    assert ctypes.sizeof(_lib.CloudDesc) == _lib.load().tcr_cloud_desc_bytes()
    assert ctypes.sizeof(_lib.BatchDesc) == _lib.load().tcr_batch_desc_bytes()
    assert _lib.load().tcr_version() == 10


def _batch(clouds, mode=0, self_search=1):
    from torchcompactradius_b200 import _lib
    arr = (_lib.CloudDesc * len(clouds))()
    for k, (dim, nq, nr) in enumerate(clouds):
        arr[k].dim = dim
        arr[k].hash_map_length = 4096
        arr[k].n_query = nq
        arr[k].n_ref = nr
        for d in range(3):
            arr[k].domain_min[d] = -1.0
            arr[k].domain_max[d] = 1.0
    b = _lib.BatchDesc()
    b.n_clouds = len(clouds)
    b.mode = mode
    b.self_search = self_search
    b.clouds = arr
    return b, arr


def test_batch_sizes_grow_with_the_clouds_and_cover_one_search():
    from torchcompactradius_b200 import _lib
    b1, keep1 = _batch([(3, 1000, 1000)])
    s1, w1 = _lib.batch_sizes(b1)
    b2, keep2 = _batch([(3, 1000, 1000), (2, 5000, 5000), (3, 0, 0)])
    s2, w2 = _lib.batch_sizes(b2)
    assert s2 > s1 and w2 > w1
    s, w = _lib.search_sizes(6000, 6000, 3)
    assert w2 <= w + 3 * 4096  # one scratch over all points, plus the per-cloud tables


def test_invalid_batch_is_rejected_without_device_work():
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    b, keep = _batch([(3, 10, 10), (4, 10, 10)])
    rc = lib.tcr_batch_sizes(ctypes.byref(b), None, None)
    assert rc == -1 and b"cloud 1" in lib.tcr_last_error()
    b, keep = _batch([(3, 10, 12)])  # a self search needs the same cloud on both sides
    assert lib.tcr_batch_sizes(ctypes.byref(b), None, None) == -1
    b, keep = _batch([(3, 10, 10)])
    b.n_clouds = 0
    assert lib.tcr_batch_sizes(ctypes.byref(b), None, None) == -1
    b, keep = _batch([(2, 10, 10)])  # positions missing
    rc = lib.tcr_batch_build_structure(ctypes.byref(b), None, 0, None, 0, None)
    assert rc == -1 and b"positions" in lib.tcr_last_error()


def test_sizes_and_layout_are_consistent():
    from torchcompactradius_b200 import _lib
    s, w = _lib.search_sizes(1 << 20, 1 << 20, 3)
    off = _lib.structure_offsets(1 << 20)
    assert off["map"] + off["map_capacity"] * 8 <= s
    assert off["map_capacity"] >= 2 * (1 << 20)
    assert all(off[k] % 256 == 0 for k in off if k != "map_capacity")
    with pytest.raises(_lib.TcrError):
        _lib.search_sizes(-1, 5, 3)


def test_invalid_descriptor_is_rejected_without_device_work():
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    d = _lib.SearchDesc()
    d.dim = 4
    rc = lib.tcr_build_structure(ctypes.byref(d), None, 0, None, 0, None)
    assert rc == -1 and b"dim" in lib.tcr_last_error()
    d.dim = 3
    d.mode = 0
    d.hash_map_length = 4096
    d.n_query = 10
    d.n_ref = 10
    rc = lib.tcr_count(ctypes.byref(d), None, None, 0, None, 0, None, None, None, None, None)
    assert rc == -1


def test_public_api_fails_loudly_without_cuda():
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import torchcompactradius_b200 as tcr
    pc = tcr.PointCloud(torch.rand(10, 2), torch.full((10,), 0.1))
    with pytest.raises(RuntimeError, match="CUDA"):
        tcr.radiusSearch(pc, algorithm="compact")


def test_api_argument_validation_matches_reference():
    import torchcompactradius_b200 as tcr
    pc = tcr.PointCloud(torch.rand(10, 2), torch.full((10,), 0.1))
    with pytest.raises(AssertionError):
        tcr.radiusSearch(pc, mode="bogus")
    with pytest.raises(AssertionError):
        tcr.radiusSearch(pc, format="dense")
    with pytest.raises(AssertionError):
        tcr.radiusSearch(pc, algorithm="cluster")
    with pytest.raises(ValueError):
        tcr.radiusSearch(pc, supportOverride=1)


def test_coo_csr_helpers():
    from torchcompactradius_b200.util import SparseCOO, coo_to_csr, csr_to_coo
    row = torch.tensor([0, 0, 2, 2, 2])
    col = torch.tensor([1, 3, 0, 1, 4])
    csr = coo_to_csr(SparseCOO(row, col, 4, 5), isSorted=True)
    assert csr.indptr.dtype == torch.int32 and csr.indptr.tolist() == [0, 2, 2, 5, 5]
    assert csr.rowEntries.dtype == torch.int64 and csr.rowEntries.tolist() == [2, 0, 3, 0]
    back = csr_to_coo(csr)
    assert back.row.tolist() == row.tolist() and back.col.tolist() == col.tolist()


def test_tuning_travels_in_the_descriptor_and_is_validated():
    """The engine keeps no tuning state: each batch descriptor carries its own, checked on use."""
    import threading

    from torchcompactradius_b200 import _lib, context, tuning
    lib = _lib.load()
    b, keep = _batch([(3, 1000, 1000)])
    s, w = ctypes.c_int64(), ctypes.c_int64()
    b.unit_queries = 12
    assert lib.tcr_batch_sizes(ctypes.byref(b), ctypes.byref(s), ctypes.byref(w)) == -1
    assert b"unit_queries" in lib.tcr_last_error()
    b.unit_queries, b.walk_blocks_per_sm = 0, 65
    assert lib.tcr_batch_sizes(ctypes.byref(b), ctypes.byref(s), ctypes.byref(w)) == -1
    b.unit_queries, b.walk_blocks_per_sm = 16, 8
    assert lib.tcr_batch_sizes(ctypes.byref(b), ctypes.byref(s), ctypes.byref(w)) == 0
    with pytest.raises(ValueError):
        tuning.set_tuning(12, 0)
    # a setting made on one thread does not reach another thread's searches
    tuning.set_tuning(16, 8)
    seen = []
    t = threading.Thread(target=lambda: seen.append(context.current().tuning()))
    t.start()
    t.join()
    assert context.current().tuning() == (16, 8) and seen == [(0, 0)]
    ctx = context.SearchContext(unit_queries=8)
    with context.use(ctx):
        d = context.apply_tuning(_lib.SearchDesc())
        assert (d.unit_queries, d.walk_blocks_per_sm) == (8, 0)
    tuning.set_tuning(0, 0)
    assert context.current().tuning() == (0, 0)


def test_scatter_descriptor_and_validation_without_device_work():
    """tcr_scatter_desc layout, scratch sizing per index layout, and argument checks that fail
    before any device call."""
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    assert ctypes.sizeof(_lib.ScatterDesc) == lib.tcr_scatter_desc_bytes()
    d = _lib.ScatterDesc()
    d.reduce, d.dtype, d.B, d.E, d.K, d.N = 0, 7, 1, 1000, 1, 50
    d.index_sorted = 1
    sorted_bytes = _lib.scatter_sizes(d)
    d.index_sorted = 0
    unsorted_bytes = _lib.scatter_sizes(d)
    assert unsorted_bytes > sorted_bytes > 0  # only an unsorted index needs the sort buffers
    d.index_full, d.B, d.K = 1, 2, 3
    assert _lib.scatter_sizes(d) > unsorted_bytes
    for field, bad in (("reduce", 5), ("dtype", 9), ("N", -1)):
        e = _lib.ScatterDesc()
        e.reduce, e.dtype, e.B, e.E, e.K, e.N = 0, 7, 1, 10, 1, 4
        setattr(e, field, bad)
        assert lib.tcr_scatter_sizes(ctypes.byref(e), None) == -1
        assert lib.tcr_scatter(ctypes.byref(e), None, 0, None, None) == -1
    e = _lib.ScatterDesc()
    e.reduce, e.dtype, e.B, e.E, e.K, e.N = 3, 7, 1, 10, 1, 4  # min without arg_out / src / index
    assert lib.tcr_scatter(ctypes.byref(e), None, 0, None, None) == -1
    assert lib.tcr_index_stats(None, -1, None, None, None) == -1


def test_scatter_index_broadcast_matches_reference_rule():
    import torch
    from torchcompactradius_b200.scatter import broadcast
    src = torch.empty(3, 5, 4)
    b = broadcast(torch.arange(5), src, 1)
    assert b.shape == src.shape and b.stride(0) == 0 and b.stride(2) == 0
    assert torch.equal(b[2, :, 3], torch.arange(5))
    full = torch.zeros(3, 5, 4, dtype=torch.int64)
    assert broadcast(full, src, 1).data_ptr() == full.data_ptr()


def test_noalloc_accepts_exactly_what_its_static_array_holds():
    """tcr_search_noalloc rejects, before any device work, every search whose structure plus
    scratch (tcr_search_sizes) exceed its 32 MiB array, naming the bytes; the largest self-search
    below the limit is sized within it."""
    from torchcompactradius_b200 import _lib
    lib = _lib.load()
    limit = 32 << 20
    for dim in (1, 2, 3):
        lo, hi = 1, 1 << 22
        while hi - lo > 1:  # largest n whose self-search fits
            mid = (lo + hi) // 2
            s, w = _lib.search_sizes(mid, mid, dim)
            lo, hi = (mid, hi) if s + w <= limit else (lo, mid)
        n = hi
        s, w = _lib.search_sizes(n, n, dim)
        assert s + w > limit
        d = _lib.SearchDesc()
        d.dim, d.mode, d.self_search, d.hash_map_length = dim, 0, 1, 4096
        d.n_query = d.n_ref = n
        for k in range(3):
            d.domain_max[k] = 1.0
        d.query_pos = d.ref_pos = d.query_sup = d.ref_sup = 256  # never dereferenced: rejected first
        total = ctypes.c_int64(-1)
        col = ctypes.c_void_p(512)
        off = ctypes.c_void_p(768)
        rc = lib.tcr_search_noalloc(ctypes.byref(d), off, None, None, None, col, 1, ctypes.byref(total), None)
        msg = lib.tcr_last_error()
        assert rc == -1 and total.value == -1
        assert b"static" in msg and str(s + w).encode() in msg
        s1, w1 = _lib.search_sizes(lo, lo, dim)
        assert s1 + w1 <= limit and lo > 50000
