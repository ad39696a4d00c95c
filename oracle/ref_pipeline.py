"""The reference's own compact search on the CPU, driven without its Python package.

Test infrastructure only (the ``reference`` CPU baseline of ``bench.py`` and a cross-check in
``tests/``).  The heavy loops -- ``countNeighbors``, ``buildNeighborList`` and
``computeHashIndices`` -- are the reference's compiled C++ operators, built from its sources by
``oracle/build_ref.py`` into ``oracle/_ref/``.  The glue between them is a line-by-line
restatement, in torch tensor operations, of the reference's Python driver (paths relative to
``src/torchCompactRadius/``):

  radiusSearch            neighborhood.py:136-309   (compact branch, explicit domain)
  neighborSearch          searchAlgorithms/compactSearch.py:12-171
  neighborSearch_cpp      compactHashing/cppSearch.py:179-244
  computeGridSupport      compactHashing/cellTable.py:40-81
  sortReferenceParticles  compactHashing/cellTable.py:7-37 with util.compute_h (util.py:28-79)
                          and util.linearIndexing (util.py:176-193)
  buildCompactHashMap_compat  compactHashing/hashTable.py:159-234
  searchNeighbors_cpp     compactHashing/cppSearch.py:12-98
  coo_to_csr              util.py:335-358
"""
import glob
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
_loaded = None


def ref_lib_path():
    c = sorted(glob.glob(os.path.join(HERE, "_ref", "torchCompactRadius_cpu*.so")))
    return c[0] if c else None


def available():
    return ref_lib_path() is not None


def ops():
    global _loaded
    if _loaded is None:
        p = ref_lib_path()
        if p is None:
            raise FileNotFoundError("oracle/_ref/torchCompactRadius_cpu.so is not built (run oracle/build_ref.py)")
        torch.ops.load_library(p)
        _loaded = torch.ops.torchCompactRadius_cpu
    return _loaded


def _wrap(x, dmin, dmax, periodic):
    # util.py:387 / cppSearch.py:221
    cols = [x[:, i] if not bool(p) else torch.remainder(x[:, i] - dmin[i], dmax[i] - dmin[i]) + dmin[i]
            for i, p in enumerate(periodic)]
    return torch.stack(cols, dim=1)


def compute_h(qMin, qMax, referenceSupport):
    # util.py:28-79
    qExtent = qMax - qMin
    qCells = qExtent / referenceSupport
    numCells = torch.floor(qCells)
    h = qExtent / numCells
    if torch.any(qExtent / h - numCells > 0):
        numCells -= 1
        h = qExtent / numCells
    if torch.any(torch.ceil(qExtent / h) > qExtent / h):
        h = h * (1e-4 + 1)
    return torch.max(h)


def _linear(ci, counts):
    # util.py:176-193
    lin = torch.zeros(ci.shape[0], dtype=ci.dtype)
    prod = 1
    for i in range(ci.shape[1]):
        lin += ci[:, i] * prod
        prod = prod * counts[i].item()
    return lin


def build_structure(x, hMax, minD, maxD, hashMapLength):
    """buildCompactHashMap_compat (hashTable.py:159-234) over already-wrapped positions x."""
    hCell = compute_h(minD, maxD, hMax)
    qExtent = maxD - minD
    cellCount = torch.ceil(qExtent / hCell).to(torch.int32)
    idx = torch.floor((x - minD) / hCell).to(torch.int32).view(-1, x.shape[1])
    lin = _linear(idx, cellCount)
    sortIndex = torch.argsort(lin)
    sortedLin = lin[sortIndex]
    sortedPositions = x[sortIndex, :]
    cellIndices, cellCounters = torch.unique_consecutive(sortedLin, return_counts=True, return_inverse=False)
    cellCounters = cellCounters.to(torch.int32)
    cumCell = torch.hstack((torch.tensor([0], dtype=cellCounters.dtype), torch.cumsum(cellCounters, dim=0)))[:-1].to(
        torch.int32)
    sortedIdx = torch.floor((sortedPositions - minD) / hCell).to(torch.int32)
    cellGrid = sortedIdx[cumCell, :]
    cellTable = torch.stack((cellIndices, cumCell, cellCounters), dim=1)
    hashed = ops().computeHashIndices(cellGrid.to(torch.int32), hashMapLength)
    hs = torch.argsort(hashed)
    hashMap, hashCounters = torch.unique_consecutive(hashed[hs], return_counts=True, return_inverse=False)
    hashCounters = hashCounters.to(torch.int32)
    sortedCellTable = torch.stack([c[hs] for c in cellTable.unbind(1)], dim=1)
    hashTable = hashMap.new_ones(hashMapLength, 2, dtype=torch.int32) * -1
    hashTable[:, 1] = 0
    hm64 = hashMap.to(torch.int64)
    hashTable[hm64, 0] = torch.hstack((torch.tensor([0], dtype=torch.int32), torch.cumsum(hashCounters, dim=0)))[:-1].to(
        torch.int32)
    hashTable[hm64, 1] = hashCounters
    return sortedPositions, hashTable, sortedCellTable.contiguous(), hCell, cellCount, sortIndex


def radius_search(xq, hq, xr, hr, dmin, dmax, periodic, mode="gather", hashMapLength=4096, fmt="coo",
                  dtype=torch.float32):
    """radiusSearch(PointCloud(xq,hq), PointCloud(xr,hr), mode=mode, domain=(dmin,dmax,periodic),
    hashMapLength=..., algorithm='compact', format=fmt) on CPU tensors of ``dtype`` (the reference's
    operators run at float or double).

    Returns ``(row, col)`` for COO or ``(indices, indptr, rowEntries)`` for CSR, exactly as the
    reference's SparseCOO / SparseCSR fields.
    """
    with torch.no_grad():
        xq = torch.as_tensor(xq, dtype=dtype)
        hq = None if hq is None else torch.as_tensor(hq, dtype=dtype)
        if xr is None:  # neighborhood.py:187-188: the query cloud doubles as the reference cloud
            xr, hr = xq, hq
        xr = torch.as_tensor(xr, dtype=dtype)
        hr = None if hr is None else torch.as_tensor(hr, dtype=dtype)
        dmin = torch.as_tensor(dmin, dtype=dtype)
        dmax = torch.as_tensor(dmax, dtype=dtype)
        periodic = torch.as_tensor(periodic, dtype=torch.bool)
        nq, nr = xq.shape[0], xr.shape[0]
        x = _wrap(xq, dmin, dmax, periodic)                  # neighborhood.py:202
        y = _wrap(xr, dmin, dmax, periodic)                  # neighborhood.py:203
        # cellTable.py:40-81
        if mode == "scatter":
            hMax = torch.max(hr)
        elif mode == "gather":
            hMax = torch.max(hq)
        else:
            hMax = torch.max(torch.max(hr), torch.max(hq))
        y2 = _wrap(y, dmin, dmax, periodic)                  # cppSearch.py:221
        sortedPositions, hashTable, cellTable, hCell, numCells, sortIndex = build_structure(
            y2, hMax, dmin, dmax, hashMapLength)
        sortedSupports = hr[sortIndex] if hr is not None else None
        o = ops()
        counts = o.countNeighbors(x, hq, 1, sortedPositions, sortedSupports, hashTable, hashMapLength, numCells,
                                  cellTable, dmin, float(hCell), dmax, dmin, periodic, mode, False)
        offsets = torch.hstack((torch.tensor([0], dtype=torch.int32), torch.cumsum(counts, dim=0).to(torch.int32)))[:-1]
        length = offsets[-1] + counts[-1] if nq > 0 else torch.tensor(0)
        i, j = o.buildNeighborList(counts, offsets, int(length.item()), x, hq, 1, sortedPositions, sortedSupports,
                                   hashTable, hashMapLength, numCells, cellTable, dmin, float(hCell), dmax, dmin,
                                   periodic, mode, False)
        j = sortIndex[j]
        if fmt == "coo":
            return i, j
        # util.py:335-358 coo_to_csr(isSorted=True)
        jj, nit = torch.unique(i, return_counts=True)
        nj = torch.zeros(nq, dtype=i.dtype)
        nj[jj] = nit
        indptr = torch.zeros(nq + 1, dtype=torch.int64)
        indptr[1:] = torch.cumsum(nj, 0)
        return j, indptr.int(), nj
