"""Host orchestration of the CUDA search through the C ABI, and the reusable structure.

One search is three C-ABI calls on torch's current stream -- ``tcr_build_structure``,
``tcr_count`` and ``tcr_emit`` -- enqueued back to back into buffers sized from the previous
search's pairs per query; the host synchronises once at the end to learn the pair count (the
reference synchronises between count and build, compactHashing/cppSearch.py:89) and re-runs
only the emit when the estimate was short.  Device memory comes from torch's caching allocator.
"""
import ctypes
import threading
import warnings
from typing import Optional

import torch

from . import _lib
from . import context as _context

_tls = threading.local()


def _info_buffer():
    buf = getattr(_tls, "info", None)
    if buf is None:
        buf = torch.zeros(8, dtype=torch.int64, pin_memory=torch.cuda.is_available())
        _tls.info = buf
    return buf


def _require_cuda(device):
    if not torch.cuda.is_available():
        raise RuntimeError("torchcompactradius_b200 runs on CUDA only and no CUDA device is available")
    if device.type != "cuda":
        device = torch.device("cuda", torch.cuda.current_device())
    return device


def _to_host(tensors):
    """Device results for a caller whose inputs live on the CPU: copied into pinned (page-locked)
    host tensors on the current stream, which then is waited for.  Pinned blocks come from torch's
    pinned-memory cache, so repeated searches reuse them; a pageable destination copies at a
    fraction of the link's rate (19 ms against 7 ms for the 0.4 GB of a 1M-point search)."""
    out = []
    for t in tensors:
        if t is None:
            out.append(None)
            continue
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        out.append(h)
    torch.cuda.current_stream().synchronize()
    return tuple(out)


_warned_f64 = False


def _as_f32(t, device, shape=None):
    """Positions and supports as contiguous float32 on the device.  The search computes in float32
    (the reference's float path); a float64 input is rounded to float32 first, with one warning per
    process, since the reference searches float64 inputs in double and pairs whose distance lies
    within float32 rounding of the threshold can then differ."""
    global _warned_f64
    t = torch.as_tensor(t)
    if t.dtype == torch.float64 and not _warned_f64:
        _warned_f64 = True
        warnings.warn("torchcompactradius_b200 searches in float32: float64 positions / supports are rounded to "
                      "float32 (pairs within float32 rounding of the threshold may differ from a float64 search)",
                      stacklevel=3)
    t = t.to(device=device, dtype=torch.float32)
    return t.contiguous()


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _domain_host(domain, dim):
    lo = [float(v) for v in torch.as_tensor(domain.min).detach().cpu().reshape(-1).tolist()]
    hi = [float(v) for v in torch.as_tensor(domain.max).detach().cpu().reshape(-1).tolist()]
    per = torch.as_tensor(domain.periodic).detach().cpu().reshape(-1).tolist()
    if isinstance(per, bool):
        per = [per] * dim
    if len(per) == 1 and dim > 1:
        per = per * dim
    if len(lo) != dim or len(hi) != dim or len(per) != dim:
        raise ValueError(f"domain has {len(lo)}/{len(hi)}/{len(per)} entries for dim {dim}")
    mask = 0
    for d, p in enumerate(per):
        if bool(p):
            mask |= 1 << d
    return lo, hi, mask


def make_desc(dim, mode, mask, lo, hi, L, xq, hq, xr, hr, self_search):
    d = _lib.SearchDesc()
    d.dim = dim
    d.mode = _lib.MODES[mode]
    d.periodic_mask = mask
    d.self_search = 1 if self_search else 0
    for k in range(3):
        d.domain_min[k] = lo[k] if k < dim else 0.0
        d.domain_max[k] = hi[k] if k < dim else 1.0
    d.hash_map_length = int(L)
    d.n_query = xq.shape[0]
    d.n_ref = xr.shape[0]
    d.query_pos = xq.data_ptr() if xq.numel() else None
    d.query_sup = hq.data_ptr() if hq is not None and hq.numel() else None
    d.ref_pos = xr.data_ptr() if xr.numel() else None
    d.ref_sup = hr.data_ptr() if hr is not None and hr.numel() else None
    return _context.apply_tuning(d)


class CompactHashMap:
    """The search structure of one reference cloud, reusable for later queries.

    Carries the fields of the reference's ``CompactHashMap`` NamedTuple
    (compactHashing/datastructure.py:8-31).  The device buffer holds the B200 layout (points in
    cell order as float4, a cell table and an open-addressing linear-index map); the
    reference-layout views (``hashTable`` [L,2], ``sortedCellTable`` [C,3], ``numCells``,
    ``hCell``, ...) are derived from it on first access.
    """

    def __init__(self, buf, n_ref, dim, lo, hi, mask, L, device, referencePositions, referenceSupports,
                 fixedSupport=None, searchRadius=1):
        self._buf = buf
        self._n = n_ref
        self._dim = dim
        self._lo, self._hi, self._mask = lo, hi, mask
        self._device = device
        self._off = _lib.structure_offsets(n_ref)
        self.hashMapLength = int(L)
        self.referencePositions = referencePositions
        self.referenceSupports = referenceSupports
        self.fixedSupport = fixedSupport
        self.searchRadius = searchRadius
        self._cache = {}
        self._f64 = None  # float64 references: their wrapped copies and cell size (search64.py)

    # -- raw device views -------------------------------------------------------------------
    def _view(self, field, dtype, count):
        off = self._off[field]
        nbytes = count * torch.empty((), dtype=dtype).element_size()
        return self._buf[off:off + nbytes].view(dtype)

    def _grid(self):
        # GridParams (include/tcr_b200.h, TCR_STRUCT_GRID): float hmax, float hCell, float hcell_d[3],
        # int32 cellCount[3], ...
        if "grid" not in self._cache:
            g = self._view("grid", torch.int32, 8).cpu()
            f = g[:5].view(torch.float32)
            self._cache["grid"] = (float(f[0]), float(f[1]), g[5:8].tolist())
        return self._cache["grid"]

    @property
    def numCellsOccupied(self):
        return int(self._view("num_cells", torch.int32, 1).item())

    # -- reference CompactHashMap fields ----------------------------------------------------
    @property
    def periodicity(self):
        return torch.tensor([bool((self._mask >> d) & 1) for d in range(self._dim)], dtype=torch.bool,
                            device=self._device)

    periodic = periodicity  # neighborhood.py:81 reads this name

    @property
    def minD(self):
        return torch.tensor(self._lo, dtype=torch.float32, device=self._device)

    @property
    def maxD(self):
        return torch.tensor(self._hi, dtype=torch.float32, device=self._device)

    qMin = minD
    qMax = maxD

    @property
    def hCell(self):
        return torch.tensor(self._grid()[1], dtype=torch.float32, device=self._device)

    @property
    def numCells(self):
        """Cells per dimension, int32 [dim] (the reference's name for cellCount)."""
        return torch.tensor(self._grid()[2][:self._dim], dtype=torch.int32, device=self._device)

    @property
    def sortedPositions(self):
        pts = self._view("sorted_points", torch.float32, 4 * self._n).view(self._n, 4)
        return pts[:, :self._dim]

    @property
    def sortedSupports(self):
        if self.referenceSupports is None:
            return None
        return self._view("sorted_points", torch.float32, 4 * self._n).view(self._n, 4)[:, 3]

    @property
    def sortIndex(self):
        return self._view("sort_index", torch.int32, self._n).to(torch.int64)

    def _reference_tables(self):
        if "tables" not in self._cache:
            C = self.numCellsOccupied
            start = self._view("cell_start", torch.int32, C + 1)
            lin = self._view("cell_lin", torch.int32, C)
            bucket = self._view("cell_bucket", torch.int32, C)
            cnt = start[1:] - start[:-1]
            order = torch.argsort(bucket, stable=True)
            table = torch.stack([lin[order], start[:-1][order], cnt[order]], dim=1).to(torch.int32)
            L = self.hashMapLength
            ht = torch.full((L, 2), -1, dtype=torch.int32, device=self._device)
            ht[:, 1] = 0
            b_sorted = bucket[order].to(torch.int64)
            if C:
                uniq, counts = torch.unique_consecutive(b_sorted, return_counts=True)
                first = torch.cumsum(counts, 0) - counts
                ht[uniq, 0] = first.to(torch.int32)
                ht[uniq, 1] = counts.to(torch.int32)
            self._cache["tables"] = (ht, table.contiguous())
        return self._cache["tables"]

    @property
    def hashTable(self):
        """int32 [hashMapLength, 2]: (first entry in sortedCellTable, entries) or (-1, 0)."""
        return self._reference_tables()[0]

    @property
    def sortedCellTable(self):
        """int32 [C, 3]: (linear index, first sorted point, points), rows grouped by hash bucket."""
        return self._reference_tables()[1]

    _fields = ("sortedPositions", "referencePositions", "hashTable", "hashMapLength", "sortedCellTable", "numCells",
               "qMin", "qMax", "minD", "maxD", "sortIndex", "hCell", "periodicity", "searchRadius", "sortedSupports",
               "referenceSupports", "fixedSupport")

    def _asdict(self):
        return {k: getattr(self, k) for k in self._fields}

    def __repr__(self):
        return f"CompactHashMap(n={self._n}, dim={self._dim}, hashMapLength={self.hashMapLength})"


def _check_device_fault(info):
    """info[1] == -1: a bounded wait inside a one-pass scan or sort gave up (the device did not make
    progress); the result is not valid."""
    if int(info[1]) < 0:
        raise RuntimeError("a device-wide scan or sort of the search did not complete (a bounded wait gave up); "
                           "the result is not valid")


def _check_info(info):
    _check_device_fault(info)
    if int(info[1]) != 0:
        raise ValueError("no valid cell grid for this domain and support (the support is not smaller than the "
                         "domain extent, or a support/domain value is not finite)")


def _scaled_cells(desc, scale, mode, hq, hr, lo, hi, mask, dim):
    """Cells `scale` times the largest threshold a pair can have (on periodic dimensions a whole
    number of cells spans the domain), searched on the clamped grid, which finds exactly the pairs
    with dist < thr for any cell at least that large.  The largest support is read from the device
    (one synchronisation)."""
    if scale < 1.0:
        raise ValueError("the cell-size multiplier must be >= 1")
    from .multilevel import GROW, cell_sizes
    parts = [t for t, use in ((hq, mode != "scatter"), (hr, mode != "gather")) if use and t is not None and t.numel()]
    if not parts:
        return
    hmax = float(torch.stack([t.max() for t in parts]).max())
    if not (hmax > 0 and hmax < float("inf")):
        return
    cells = cell_sizes(scale * hmax * GROW, lo, hi, mask, dim)
    for d in range(3):
        desc.hcell[d] = cells[d] if d < dim else 1.0
    desc.clamped_grid = 1


def compact_search(xq, hq, xr, hr, domain_lo, domain_hi, mask, mode, L, fmt, self_search, return_structure=False,
                   structure: Optional[CompactHashMap] = None, ref_pos_user=None, ref_sup_user=None,
                   fixed_support=None, events=None):
    """Runs one search on the current CUDA stream.  xq/hq/xr/hr are contiguous float32 device
    tensors (hq/hr may be None when the mode does not read them).  Returns (i, j) for COO or
    (indices, indptr, rowEntries) for CSR, plus the structure when asked.

    ``events``: optional dict that receives CUDA event pairs bracketing the 'build', 'count' and
    'emit' phases on the launching stream (for benchmarks)."""
    lib = _lib.load()
    device = xq.device
    dim = xq.shape[1]
    nq, nr = xq.shape[0], xr.shape[0]
    stream = torch.cuda.current_stream(device)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    desc = make_desc(dim, mode, mask, domain_lo, domain_hi, L, xq, hq, xr, hr, self_search)
    scale = float(_context.current().cell_scale)
    if scale != 1.0 and structure is None and not return_structure:
        _scaled_cells(desc, scale, mode, hq, hr, domain_lo, domain_hi, mask, dim)
    s_bytes, w_bytes = _lib.search_sizes(nq, nr, dim)
    scratch = torch.empty(w_bytes, dtype=torch.uint8, device=device)
    def mark(name, end=False):
        if events is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            events.setdefault(name, [None, None])[1 if end else 0] = ev

    if structure is None:
        sbuf = torch.empty(s_bytes, dtype=torch.uint8, device=device)
        mark("build")
        _lib.check(lib.tcr_build_structure(ctypes.byref(desc), _ptr(sbuf), s_bytes, _ptr(scratch), w_bytes, sptr),
                   "tcr_build_structure")
        mark("build", True)
        if return_structure:
            structure = CompactHashMap(sbuf, nr, dim, domain_lo, domain_hi, mask, L, device,
                                       ref_pos_user if ref_pos_user is not None else xr,
                                       ref_sup_user if ref_sup_user is not None else hr, fixed_support)
    else:
        sbuf = structure._buf
    offsets = torch.empty(nq + 1, dtype=torch.int64, device=device)
    indptr = rowEntries = None
    if fmt == "csr":
        indptr = torch.empty(nq + 1, dtype=torch.int32, device=device)
        rowEntries = torch.empty(nq, dtype=torch.int64, device=device)
    info = _info_buffer()
    # One estimate sizes both the staging list and the output, so count and emit are enqueued
    # back to back and the host waits only once, at the end.
    ctx = _context.current()
    cap = int(min(0x7fffffff, ctx.pairs_per_query * 1.25 * nq + 4096))
    stage_cap = int(min(0x7fffffff, ctx.stage_per_query * 1.1 * nq + 65536))
    stage = torch.empty(stage_cap, dtype=torch.int32, device=device)
    col = torch.empty(cap, dtype=torch.int64, device=device)
    row = torch.empty(cap, dtype=torch.int64, device=device) if fmt == "coo" else None
    mark("count")
    _lib.check(lib.tcr_count(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), stage_cap,
                             _ptr(offsets), _ptr(indptr), _ptr(rowEntries), ctypes.c_void_p(info.data_ptr()), sptr),
               "tcr_count")
    mark("count", True)
    mark("emit")
    _lib.check(lib.tcr_emit(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), _ptr(offsets),
                            _ptr(row), _ptr(col), cap, sptr), "tcr_emit")
    mark("emit", True)
    stream.synchronize()
    _check_info(info)
    total = int(info[0])
    if nq:
        ctx.pairs_per_query = max(total / nq, 1.0)
        ctx.stage_per_query = max(int(info[4]) / nq, 1.0)
    if fmt == "csr" and total > 0x7fffffff:
        raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
    if total > cap:  # the estimate was short: emit again into an exact buffer (the count is kept)
        col = torch.empty(total, dtype=torch.int64, device=device)
        row = torch.empty(total, dtype=torch.int64, device=device) if fmt == "coo" else None
        _lib.check(lib.tcr_emit(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), _ptr(offsets),
                                _ptr(row), _ptr(col), total, sptr), "tcr_emit")
    col = col[:total]
    row = row[:total] if row is not None else None
    out = (row, col) if fmt == "coo" else (col, indptr, rowEntries)
    return out, structure
