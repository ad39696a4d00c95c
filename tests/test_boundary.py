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
    assert _lib.load().tcr_version() == 5


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
