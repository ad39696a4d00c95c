"""B200-native (sm_100a) compact-hashing fixed-radius neighbour search.

A drop-in for torchCompactRadius's ``radiusSearch`` / ``radius`` / ``neighborSearchExisting``
API (same types, arguments and outputs), and of its scatter_sum / scatter_mul / scatter_mean /
scatter_min / scatter_max operators, computed by hand-written CUDA kernels behind a C ABI
(include/tcr_b200.h).  There is no CPU fallback.
"""
from .batched import BatchedAdjacency, radiusSearchBatch
from .neighborhood import neighborSearchExisting, radius, radiusSearch
from .scatter import scatter_max, scatter_mean, scatter_min, scatter_mul, scatter_sum
from .search import CompactHashMap
from .util import (DomainDescription, PointCloud, SparseCOO, SparseCSR, coo_to_csr, csr_to_coo,
                   getPeriodicPointCloud, volumeToSupport)

__version__ = "0.1.0"
__all__ = ["radiusSearch", "radiusSearchBatch", "BatchedAdjacency", "radius", "neighborSearchExisting", "volumeToSupport",
           "PointCloud", "DomainDescription", "SparseCOO", "SparseCSR", "CompactHashMap", "coo_to_csr", "csr_to_coo",
           "getPeriodicPointCloud", "scatter_sum", "scatter_mul", "scatter_mean", "scatter_min", "scatter_max"]
