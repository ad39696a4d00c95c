"""The TORCH_LIBRARY operator layer (csrc/tcr_torch_ops.cpp): registration and schemas on CPU;
the reference-schema operators and the fused / split / batched forms against the C oracle on the
GPU.  The reference's own operators are bound as torch.ops.torchCompactRadius_cuda.countNeighbors /
buildNeighborList (compactHashing/cppWrapper.py:10-65); these tests call torch.ops.tcr_b200.* with
the same argument lists (cppSrc/neighborhood.h:102-124)."""
import hashlib

import numpy as np
import pytest
import torch

from oracle import compact


def _digest(row, col, ncols):
    key = np.asarray(row, np.int64) * np.int64(max(int(ncols), 1)) + np.asarray(col, np.int64)
    key.sort()
    return hashlib.sha256(key.tobytes()).hexdigest(), len(key)


def test_operators_register_with_the_reference_schemas():
    from torchcompactradius_b200 import ops
    ns = ops.load()
    s = str(ns.countNeighbors.default._schema)
    assert s.startswith("tcr_b200::countNeighbors(Tensor queryPositions, Tensor querySupport, int searchRange, "
                        "Tensor sortedPositions, Tensor sortedSupport, Tensor hashTable, int hashMapLength, "
                        "Tensor numCells, Tensor cellTable, Tensor qMin, float hCell, Tensor maxDomain, "
                        "Tensor minDomain, Tensor periodicity, str mode, bool verbose=False) -> Tensor")
    s = str(ns.buildNeighborList.default._schema)
    assert "int neighborListLength" in s and s.endswith("-> (Tensor, Tensor)")
    for name in ("radiusSearch", "buildStructure", "radiusSearchWithStructure", "radiusSearchBatched"):
        assert hasattr(ns, name)


def test_operators_have_no_cpu_implementation():
    from torchcompactradius_b200 import ops
    ns = ops.load()
    x = torch.rand(10, 2)
    with pytest.raises((NotImplementedError, RuntimeError)):
        ns.radiusSearch(x, torch.full((10,), 0.1), x, None, torch.zeros(2), torch.ones(2),
                        torch.tensor([False, False]), 4096, "gather", True)


def _cloud(seed, n, dim, h, per):
    rng = np.random.default_rng(seed)
    x = (rng.random((n, dim)) * 2 - 1).astype(np.float32)
    hx = (h * (0.8 + 0.4 * rng.random(n))).astype(np.float32)
    lo, hi = np.full(dim, -1.0, np.float32), np.full(dim, 1.0, np.float32)
    return x, hx, lo, hi, np.array(per)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["gather", "scatter", "symmetric", "superSymmetric"])
@pytest.mark.parametrize("dim,per", [(2, [True, False]), (3, [False, False, False]), (3, [True, True, True])])
def test_reference_schema_operators_match_the_oracle(mode, dim, per):
    from torchcompactradius_b200 import ops
    ns = ops.load()
    x, hx, lo, hi, p = _cloud(5 + dim, 20000, dim, 0.05 if dim == 2 else 0.09, per)
    y, hy, _, _, _ = _cloud(50 + dim, 15000, dim, 0.05 if dim == 2 else 0.09, per)
    # the reference's call of cppSearch.py:74-95: queries against a (sorted) reference cloud
    perm = np.random.default_rng(1).permutation(len(y))
    ys, hys = y[perm], hy[perm]
    dev = torch.device("cuda")
    xq, hq = torch.tensor(x, device=dev), torch.tensor(hx, device=dev)
    xs, hs = torch.tensor(ys, device=dev), torch.tensor(hys, device=dev)
    minD, maxD = torch.tensor(lo, device=dev), torch.tensor(hi, device=dev)
    pt = torch.tensor(per, device=dev)
    dummy = torch.zeros(1, dtype=torch.int32, device=dev)
    counts = ns.countNeighbors(xq, hq, 1, xs, hs, dummy, 4096, dummy, dummy, minD, 0.0, maxD, minD, pt, mode, False)
    o = compact.radius_search(x, hx, ys, hys, lo, hi, p, mode, 4096)
    assert counts.dtype == torch.int32
    np.testing.assert_array_equal(counts.cpu().numpy(), o.counts)
    offs = torch.cumsum(counts, 0, dtype=torch.int32) - counts
    total = int(counts.sum())
    i, j = ns.buildNeighborList(counts, offs, total, xq, hq, 1, xs, hs, dummy, 4096, dummy, dummy, minD, 0.0, maxD,
                                minD, pt, mode, False)
    assert i.dtype == torch.int64 and j.dtype == torch.int64
    assert bool((i[1:] >= i[:-1]).all())  # rows in query order, as the reference's list
    assert _digest(i.cpu().numpy(), j.cpu().numpy(), len(y)) == _digest(o.row, o.col, len(y))
    with pytest.raises(RuntimeError, match="neighborListLength"):
        ns.buildNeighborList(counts, offs, total + 1, xq, hq, 1, xs, hs, dummy, 4096, dummy, dummy, minD, 0.0, maxD,
                             minD, pt, mode, False)


@pytest.mark.gpu
def test_fused_split_and_batched_operators_match_the_oracle():
    from torchcompactradius_b200 import ops
    ns = ops.load()
    dev = torch.device("cuda")
    x, hx, lo, hi, p = _cloud(3, 30000, 3, 0.08, [True, False, True])
    xt, ht = torch.tensor(x, device=dev), torch.tensor(hx, device=dev)
    minD, maxD, pt = torch.tensor(lo), torch.tensor(hi), torch.tensor(p)
    o = compact.radius_search(x, hx, None, None, lo, hi, p, "symmetric", 4096)
    row, col, off = ns.radiusSearch(xt, ht, xt, ht, minD, maxD, pt, 4096, "symmetric", True)
    assert _digest(row.cpu().numpy(), col.cpu().numpy(), len(x)) == _digest(o.row, o.col, len(x))
    np.testing.assert_array_equal(torch.diff(off).cpu().numpy(), o.counts)
    # structure reuse: the same reference cloud against two query sets
    s = ns.buildStructure(xt, ht, xt, ht, minD, maxD, pt, 4096, "gather", False)
    for seed in (7, 8):
        q, hq, _, _, _ = _cloud(seed, 5000, 3, 0.08, [True, False, True])
        qt, hqt = torch.tensor(q, device=dev), torch.tensor(hq, device=dev)
        r, c, _ = ns.radiusSearchWithStructure(s, qt, hqt, xt, ht, minD, maxD, pt, 4096, "gather", False)
        og = compact.radius_search(q, hq, x, hx, lo, hi, p, "gather", 4096)
        assert _digest(r.cpu().numpy(), c.cpu().numpy(), len(x)) == _digest(og.row, og.col, len(x))
    # batched: three clouds as consecutive segments, local indices
    sizes = [4000, 9000, 17000]
    r, c, off = ns.radiusSearchBatched(xt, ht, xt, ht, torch.tensor(sizes), torch.tensor(sizes), minD, maxD, pt, 4096,
                                       "symmetric", True, True)
    offs = off.cpu().numpy()
    q0 = 0
    for n in sizes:
        ob = compact.radius_search(x[q0:q0 + n], hx[q0:q0 + n], None, None, lo, hi, p, "symmetric", 4096)
        a, b = int(offs[q0]), int(offs[q0 + n])
        assert _digest(r[a:b].cpu().numpy(), c[a:b].cpu().numpy(), n) == _digest(ob.row, ob.col, n)
        q0 += n
