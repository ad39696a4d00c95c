"""Data types and helpers with the reference's names and field layout.

Mirrors src/torchCompactRadius/util.py: ``DomainDescription`` (:280-292), ``PointCloud``
(:294-305), ``SparseCOO`` (:308-318), ``SparseCSR`` (:321-333), ``coo_to_csr`` (:335-358),
``csr_to_coo`` (:360-369), ``getPeriodicPointCloud`` (:375-387) and ``volumeToSupport`` (:5-26).
"""
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch


@dataclass
class DomainDescription:
    """Axis-aligned domain [min, max] with per-dimension periodicity."""
    min: torch.Tensor
    max: torch.Tensor
    periodic: torch.Tensor
    dim: int

    @property
    def periodicity(self):  # the name the reference README uses
        return self.periodic


@dataclass
class PointCloud:
    positions: torch.Tensor
    supports: Optional[torch.Tensor] = None


@dataclass
class SparseCOO:
    """Neighbour pairs: row = query index, col = reference index (int64), rows ascending."""
    row: torch.Tensor
    col: torch.Tensor
    numRows: int
    numCols: int


@dataclass
class SparseCSR:
    """indices int64 [P], indptr int32 [numRows+1], rowEntries int64 [numRows]."""
    indices: torch.Tensor
    indptr: torch.Tensor
    rowEntries: torch.Tensor
    numRows: int
    numCols: int


def volumeToSupport(volume: float, targetNeighbors: int, dim: int):
    """Support radius holding ``targetNeighbors`` particles of volume ``volume`` (util.py:5-26)."""
    if dim == 1:
        return targetNeighbors * volume / 2
    if dim == 2:
        return torch.sqrt(torch.as_tensor(targetNeighbors * volume / np.pi))
    return torch.pow(torch.as_tensor(targetNeighbors * volume / np.pi * 3 / 4), 1 / 3)


def coo_to_csr(coo: SparseCOO, isSorted: bool = False) -> SparseCSR:
    """util.py:335-358: int64 rowEntries, int32 indptr; indices keep the pairs' order."""
    if not isSorted:
        order = torch.argsort(coo.row, stable=True)
        row, col = coo.row[order], coo.col[order]
    else:
        row, col = coo.row, coo.col
    nj = torch.bincount(row, minlength=coo.numRows).to(coo.row.dtype) if row.numel() else torch.zeros(
        coo.numRows, dtype=coo.row.dtype, device=coo.row.device)
    indptr = torch.zeros(coo.numRows + 1, dtype=torch.int64, device=coo.row.device)
    indptr[1:] = torch.cumsum(nj, 0)
    return SparseCSR(col, indptr.int(), nj, coo.numRows, coo.numCols)


def csr_to_coo(csr: SparseCSR) -> SparseCOO:
    """util.py:360-369."""
    row = torch.repeat_interleave(torch.arange(csr.numRows, device=csr.indices.device), csr.rowEntries.to(torch.int64))
    return SparseCOO(row, csr.indices, csr.numRows, csr.numCols)


def getPeriodicPointCloud(queryPointCloud: PointCloud, domain: Optional[DomainDescription] = None):
    """util.py:375-387: remainder-wrap the periodic dimensions (torch float32 semantics)."""
    if domain is None:
        return queryPointCloud
    cols = [queryPointCloud.positions[:, i] if not bool(p) else
            torch.remainder(queryPointCloud.positions[:, i] - domain.min[i], domain.max[i] - domain.min[i]) + domain.min[i]
            for i, p in enumerate(domain.periodic)]
    return PointCloud(torch.stack(cols, dim=1), queryPointCloud.supports)
