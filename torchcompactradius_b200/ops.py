"""The search as PyTorch operators: ``torch.ops.tcr_b200.*`` (csrc/tcr_torch_ops.cpp).

``load()`` registers the operator library ``libtcr_torch_ops.so`` (built in-tree next to
``libtcr_b200.so``, whose C ABI it calls) and returns ``torch.ops.tcr_b200``:

* ``countNeighbors`` / ``buildNeighborList`` -- the schemas of the reference's operators
  (cppSrc/neighborhood.h:102-124, cppWrapper.cpp:38-40), for callers that bind
  ``torch.ops.torchCompactRadius_cuda.*`` (compactHashing/cppWrapper.py:10-65);
* ``radiusSearch`` -- the fused search (structure, count, emit; one host sync), returning
  ``(row, col, offsets)``;
* ``buildStructure`` / ``radiusSearchWithStructure`` -- the same split for structure reuse;
* ``radiusSearchBatched`` -- independent clouds, given as consecutive segments, in one search.

Every operator runs on torch's current CUDA stream and allocates through torch's caching
allocator.  There is no CPU implementation: a missing library or device raises.
"""
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
OPS_PATH = os.path.join(HERE, "libtcr_torch_ops.so")

_lock = threading.Lock()
_loaded = False


def load():
    """Registers the operators (once per process) and returns the ``torch.ops.tcr_b200`` namespace."""
    global _loaded
    with _lock:
        if not _loaded:
            if not os.path.exists(OPS_PATH):
                raise RuntimeError(f"{OPS_PATH} is missing: build it with python -m torchcompactradius_b200.build --ops")
            torch.ops.load_library(OPS_PATH)
            _loaded = True
    return torch.ops.tcr_b200
