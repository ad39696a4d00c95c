"""Float64 inputs: the reference's double search on the device.

The reference's operators dispatch on float and double (cppSrc/neighborhoodDynamic_cpu.cpp:504,531):
for float64 positions its grid, its periodic wrap and every distance test are double.  This module
keeps that arithmetic where it decides pairs and uses float32 only to find candidates:

* positions are wrapped in double exactly as the reference wraps them -- queries once
  (util.py:375-387), references twice (that, then compactHashing/cppSearch.py:221) -- with the
  same torch operation, ``remainder(x - min, max - min) + min``;
* the reference's cell size is computed in double (``compute_h``, util.py:28-79, on the mode's
  maximum support, compactHashing/cellTable.py:40-81), then rounded up to float32 and padded by a
  few float32 ulps of the largest coordinate, so that the float32 cell of every point is at least
  as wide as the double one: every pair within the double support lies in a query's 3^d stencil;
* the float32 structure is built by ``tcr_build_structure`` with that cell size, and
  ``tcr_count_f64`` / ``tcr_emit_f64`` decide every stencil candidate on the double arrays (the
  references gathered once into cell order) with the reference's double expression
  (common.h:106-129 at scalar_t = double).

The pair set is the reference's wherever the two grids have the same number of cells per periodic
dimension (they differ only for a domain extent within a few ulps of a whole number of cells).
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from . import context as _context
from .search import _check_info, _info_buffer, _ptr, make_desc


def wrap64(x: torch.Tensor, lo, hi, mask: int) -> torch.Tensor:
    """util.py:375-387: periodic columns become remainder(x - min, max - min) + min (float64)."""
    cols = []
    for d in range(x.shape[1]):
        if (mask >> d) & 1:
            cols.append(torch.remainder(x[:, d] - lo[d], hi[d] - lo[d]) + lo[d])
        else:
            cols.append(x[:, d])
    return torch.stack(cols, dim=1).contiguous()


def compute_h64(lo, hi, hmax: float) -> float:
    """util.py:28-79 in double: cells = floor(extent / hMax), h = extent / cells, one cell fewer
    when extent / h exceeds the cell count, h * (1 + 1e-4) when ceil(extent / h) > extent / h, and
    the largest h over the dimensions (NaN propagates, as torch.max does)."""
    ext = np.asarray(hi, np.float64) - np.asarray(lo, np.float64)
    with np.errstate(all="ignore"):
        cells = np.floor(ext / np.float64(hmax))
        h = ext / cells
        if np.any(ext / h - cells > 0):
            cells = cells - 1
            h = ext / cells
        if np.any(np.ceil(ext / h) > ext / h):
            h = h * (1e-4 + 1)
    if np.any(np.isnan(h)):
        return float("nan")
    return float(np.max(h))


def grid_support64(hq, hr, mode: str) -> float:
    """cellTable.py:40-81: the largest support the mode reads."""
    if mode == "scatter":
        return float(hr.max())
    if mode == "gather":
        return float(hq.max())
    return max(float(hr.max()), float(hq.max()))


def compact_search_f64(xq, hq, xr, hr, lo, hi, mask, mode, L, fmt, self_search, return_structure=False,
                       structure=None, ref_pos_user=None, fixed_support=None):
    """One float64 search on the current CUDA stream.  xq / xr are float64 device tensors (the
    caller's positions, unwrapped), hq / hr float64 or None.  Returns ((i, j) for COO or
    (indices, indptr, rowEntries) for CSR, structure): with ``return_structure`` a
    ``CompactHashMap`` that ``structure=`` (and ``neighborSearchExisting``) reuses for new
    float64 queries against the same references (then xr / hr are ignored)."""
    from .search import CompactHashMap
    lib = _lib.load()
    device = xq.device
    dim = xq.shape[1]
    nq = xq.shape[0]
    stream = torch.cuda.current_stream(device)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    xq_w = wrap64(xq, lo, hi, mask)
    if structure is not None:  # references, cell size and float32 copies of an earlier build
        f = structure._f64
        xr_w, hr, xr_f, hr_f, hcell = f["xr_w"], f["hr"], f["xr_f"], f["hr_f"], f["hcell"]
        self_search = False
    else:
        xr_w = wrap64(wrap64(xr, lo, hi, mask), lo, hi, mask)
    nr = xr_w.shape[0]
    if structure is None:
        hc = compute_h64(lo, hi, grid_support64(hq, hr, mode)) if nq and nr else 1.0
        if not (math.isfinite(hc) and hc > 0.0):
            raise ValueError("no valid cell grid for this domain and support (the support is not smaller than the "
                             "domain extent, or a support/domain value is not finite)")
        big = max([abs(v) for v in lo] + [abs(v) for v in hi] +
                  [float(t.abs().max()) for t in (xq_w, xr_w) if t.numel()])
        padded = hc + 8.0 * 2.0 ** -24 * big
        hcell = np.float32(padded)
        if float(hcell) < padded:
            hcell = np.nextafter(hcell, np.float32(np.inf))
    xq_f = xq_w.float().contiguous()
    hq_f = None if hq is None else hq.float().contiguous()
    if structure is None:
        xr_f = xq_f if self_search else xr_w.float().contiguous()
        hr_f = None if hr is None else (hq_f if (self_search and hq is hr) else hr.float().contiguous())
    desc = make_desc(dim, mode, mask, lo, hi, L, xq_f, hq_f, xr_f, hr_f, self_search)
    for k in range(dim):
        desc.hcell[k] = float(hcell)
    inputs = _lib.F64Inputs()
    inputs.query_pos = xq_w.data_ptr() if nq else None
    inputs.query_sup = None if hq is None or not nq else hq.data_ptr()
    inputs.ref_pos = xr_w.data_ptr() if nr else None
    inputs.ref_sup = None if hr is None or not nr else hr.data_ptr()
    ref_sorted = torch.empty((max(nr, 1), 4), dtype=torch.float64, device=device)
    inputs.ref_sorted = ref_sorted.data_ptr()
    for k in range(3):
        inputs.domain_min[k] = lo[k] if k < dim else 0.0
        inputs.domain_max[k] = hi[k] if k < dim else 1.0
    s_bytes, w_bytes = _lib.search_sizes(nq, nr, dim)
    scratch = torch.empty(w_bytes, dtype=torch.uint8, device=device)
    if structure is None:
        sbuf = torch.empty(s_bytes, dtype=torch.uint8, device=device)
        _lib.check(lib.tcr_build_structure(ctypes.byref(desc), _ptr(sbuf), s_bytes, _ptr(scratch), w_bytes, sptr),
                   "tcr_build_structure")
        if return_structure:
            structure = CompactHashMap(sbuf, nr, dim, lo, hi, mask, L, device,
                                       ref_pos_user if ref_pos_user is not None else xr, hr, fixed_support)
            structure._f64 = dict(xr_w=xr_w, hr=hr, xr_f=xr_f, hr_f=hr_f, hcell=hcell)
    else:
        sbuf = structure._buf
    offsets = torch.empty(nq + 1, dtype=torch.int64, device=device)
    indptr = rowEntries = None
    if fmt == "csr":
        indptr = torch.empty(nq + 1, dtype=torch.int32, device=device)
        rowEntries = torch.empty(nq, dtype=torch.int64, device=device)
    info = _info_buffer()
    # the count walk stages each unit's hit masks for the emit (sized like the float32 search's)
    ctx = _context.current()
    stage_cap = int(min(0x7fffffff, ctx.stage_per_query * 1.1 * nq + 65536))
    stage = torch.empty(stage_cap, dtype=torch.int32, device=device)
    _lib.check(lib.tcr_count_f64(ctypes.byref(desc), ctypes.byref(inputs), _ptr(sbuf), _ptr(scratch), w_bytes,
                                 _ptr(stage), stage_cap, _ptr(offsets), _ptr(indptr), _ptr(rowEntries),
                                 ctypes.c_void_p(info.data_ptr()), sptr), "tcr_count_f64")
    stream.synchronize()
    _check_info(info)
    total = int(info[0])
    if nq:
        ctx.stage_per_query = max(int(info[4]) / nq, 1.0)
    if fmt == "csr" and total > 0x7fffffff:
        raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
    col = torch.empty(max(total, 1), dtype=torch.int64, device=device)
    row = torch.empty(max(total, 1), dtype=torch.int64, device=device) if fmt == "coo" else None
    _lib.check(lib.tcr_emit_f64(ctypes.byref(desc), ctypes.byref(inputs), _ptr(sbuf), _ptr(scratch), w_bytes,
                                _ptr(stage), _ptr(offsets), _ptr(row), _ptr(col), total, sptr), "tcr_emit_f64")
    col = col[:total]
    row = row[:total] if row is not None else None
    return ((row, col) if fmt == "coo" else (col, indptr, rowEntries)), structure
