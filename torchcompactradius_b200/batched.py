"""Batched searches: many independent point clouds in one set of launches.

A batch is the many scenes or timesteps of an SPH training set or simulation sweep: clouds of
uneven sizes, each with its own domain, periodicity, supports and hashMapLength, searched
independently.  The reference runs them one call at a time (its ``radius`` with ``batch_x`` /
``batch_y``, src/torchCompactRadius/neighborhood.py:313-363, searches each batch id on its own).
Here one ``tcr_batch_*`` sequence (include/tcr_b200.h) sorts every cloud's points by (cloud, cell)
in one radix sort, builds one cell table with a map region per cloud and walks every cloud's
work units in one launch, so a batch costs the launches of one search.

The cloud table is a numpy structured array with the layout of ``tcr_cloud_desc``; building it
is vectorised, so a batch of thousands of clouds costs no per-cloud Python work beyond what the
caller's inputs need.
"""
import ctypes
from typing import List, Optional, Sequence, Union

import numpy as np
import torch

from . import _lib
from . import context as _context
from .search import _as_f32, _check_device_fault, _domain_host, _ptr, _require_cuda, _to_host
from .util import DomainDescription, PointCloud, SparseCOO, SparseCSR

CLOUD_DTYPE = np.dtype([("dim", "<i4"), ("periodic_mask", "<i4"), ("domain_min", "<f4", (3,)),
                        ("domain_max", "<f4", (3,)), ("hash_map_length", "<i8"), ("n_query", "<i8"),
                        ("n_ref", "<i8"), ("query_pos", "<u8"), ("query_sup", "<u8"), ("ref_pos", "<u8"),
                        ("ref_sup", "<u8"), ("hcell", "<f4", (3,)), ("clamped_grid", "<i4"), ("reserved", "<i4")],
                       align=True)


def cloud_table(n):
    """An empty cloud table of n entries (domain [0, 1]^3, hashMapLength 4096)."""
    t = np.zeros(n, dtype=CLOUD_DTYPE)
    t["domain_max"] = 1.0
    t["hash_map_length"] = 4096
    return t


def batch_desc(table, mode, self_search, local_index=True, query_ids=None, ref_ids=None, lin_hint=None,
               lin_out=None, order_out=None):
    """tcr_batch_desc over a cloud table (the table must stay alive while the descriptor is used).
    lin_hint / lin_out / order_out: the incremental re-sort arrays of include/tcr_b200.h."""
    if table.dtype != CLOUD_DTYPE or not table.flags["C_CONTIGUOUS"]:
        raise TypeError("the cloud table must be a contiguous CLOUD_DTYPE array")
    if CLOUD_DTYPE.itemsize != _lib.load().tcr_cloud_desc_bytes():
        raise RuntimeError("tcr_cloud_desc layout mismatch between numpy and the library")
    b = _lib.BatchDesc()
    b.n_clouds = len(table)
    b.mode = _lib.MODES[mode]
    b.self_search = 1 if self_search else 0
    b.local_index = 1 if local_index else 0
    b.clouds = ctypes.cast(table.ctypes.data, ctypes.POINTER(_lib.CloudDesc))
    b.query_ids = None if query_ids is None else query_ids.data_ptr()
    b.ref_ids = None if ref_ids is None else ref_ids.data_ptr()
    b.ref_lin_hint = None if lin_hint is None else lin_hint.data_ptr()
    b.ref_lin_out = None if lin_out is None else lin_out.data_ptr()
    b.ref_order_out = None if order_out is None else order_out.data_ptr()
    return _context.apply_tuning(b)


class BatchBuffers:
    """Device buffers of one batched search, reusable by later searches of no larger size."""

    def __init__(self, device):
        self.device = device
        self._bufs = {}

    def get(self, name, numel, dtype):
        t = self._bufs.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = torch.empty(max(numel, 1), dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t[:numel]


def run_batch(table, mode, self_search, fmt, device, local_index=True, query_ids=None, ref_ids=None,
              buffers: Optional[BatchBuffers] = None, events=None, stream=None, lin_hint=None, lin_out=None,
              order_out=None, fresh_outputs=False):
    """Runs build, count and emit of one batch on `stream` (default: torch's current stream) and
    synchronises once.  Returns a dict with the global outputs: ``row`` (COO) or None, ``col``,
    ``offsets`` (int64 [Nq+1]), ``indptr`` (int32, CSR) or None, ``counts`` (int64 [Nq]), ``total``.
    """
    lib = _lib.load()
    b = batch_desc(table, mode, self_search, local_index, query_ids, ref_ids, lin_hint, lin_out, order_out)
    s_bytes, w_bytes = _lib.batch_sizes(b)
    nq = int(table["n_query"].sum())
    stream = stream or torch.cuda.current_stream(device)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    bufs = buffers or BatchBuffers(device)
    sbuf = bufs.get("structure", s_bytes, torch.uint8)
    scratch = bufs.get("scratch", w_bytes, torch.uint8)
    offsets = bufs.get("offsets", nq + 1, torch.int64)
    counts = bufs.get("counts", nq, torch.int64)
    indptr = bufs.get("indptr", nq + 1, torch.int32) if fmt == "csr" else None
    ctx = _context.current()
    cap = int(min(0x7fffffff, ctx.batch_pairs_per_query * 1.25 * nq + 4096))
    stage_cap = int(min(0x7fffffff, ctx.batch_stage_per_query * 1.1 * nq + 65536))
    stage = bufs.get("stage", stage_cap, torch.int32)
    if fresh_outputs:  # outputs owned by the caller, not reused by the next search on these buffers
        offsets = torch.empty(nq + 1, dtype=torch.int64, device=device)
        counts = torch.empty(max(nq, 0), dtype=torch.int64, device=device)
        indptr = torch.empty(nq + 1, dtype=torch.int32, device=device) if fmt == "csr" else None
        col = torch.empty(cap, dtype=torch.int64, device=device)
        row = torch.empty(cap, dtype=torch.int64, device=device) if fmt == "coo" else None
    else:
        col = bufs.get("col", cap, torch.int64)
        row = bufs.get("row", cap, torch.int64) if fmt == "coo" else None
    info = bufs._bufs.get("info")
    if info is None:
        info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
        bufs._bufs["info"] = info

    def mark(name, end=False):
        if events is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            events.setdefault(name, [None, None])[1 if end else 0] = ev

    mark("build")
    _lib.check(lib.tcr_batch_build_structure(ctypes.byref(b), _ptr(sbuf), s_bytes, _ptr(scratch), w_bytes, sptr),
               "tcr_batch_build_structure")
    mark("build", True)
    mark("count")
    _lib.check(lib.tcr_batch_count(ctypes.byref(b), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), stage_cap,
                                   _ptr(offsets), _ptr(indptr), _ptr(counts), ctypes.c_void_p(info.data_ptr()),
                                   sptr), "tcr_batch_count")
    mark("count", True)
    mark("emit")
    _lib.check(lib.tcr_batch_emit(ctypes.byref(b), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), _ptr(offsets),
                                  _ptr(row), _ptr(col), cap, sptr), "tcr_batch_emit")
    mark("emit", True)
    stream.synchronize()
    _check_device_fault(info)
    if int(info[1]) != 0:
        raise ValueError(f"{int(info[1])} cloud(s) have no valid cell grid for their domain and support (the "
                         "support is not smaller than the domain extent, or a support/domain value is not finite)")
    total = int(info[0])
    if nq:
        ctx.batch_pairs_per_query = max(total / nq, 1.0)
        ctx.batch_stage_per_query = max(int(info[4]) / nq, 1.0)
    if fmt == "csr" and total > 0x7fffffff:
        raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
    if total > cap:  # the estimate was short: emit again into exact buffers (the count is kept)
        if fresh_outputs:
            col = torch.empty(total, dtype=torch.int64, device=device)
            row = torch.empty(total, dtype=torch.int64, device=device) if fmt == "coo" else None
        else:
            col = bufs.get("col", total, torch.int64)
            row = bufs.get("row", total, torch.int64) if fmt == "coo" else None
        _lib.check(lib.tcr_batch_emit(ctypes.byref(b), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage),
                                      _ptr(offsets), _ptr(row), _ptr(col), total, sptr), "tcr_batch_emit")
    return dict(row=None if row is None else row[:total], col=col[:total], offsets=offsets, indptr=indptr,
                counts=counts, total=total, info=info.clone())


class PendingBatch:
    """A batched search enqueued on a stream and not waited for (``enqueue_batch``).  It owns every
    buffer its kernels use until ``finish()``, which waits for ``event`` (recorded after the emit),
    checks the device's info block and, when the output estimate was short, emits again into exact
    buffers -- the count, offsets and staging list are kept, so only the emit runs twice."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def finish(self):
        self.event.synchronize()
        info = self.info
        _check_device_fault(info)
        if int(info[1]) != 0:
            raise ValueError(f"{int(info[1])} cloud(s) have no valid cell grid for their domain and support")
        total = int(info[0])
        if total > self.cap:
            lib = _lib.load()
            self.col = torch.empty(total, dtype=torch.int64, device=self.device)
            self.row = torch.empty(total, dtype=torch.int64, device=self.device) if self.fmt == "coo" else None
            sptr = ctypes.c_void_p(self.stream.cuda_stream)
            _lib.check(lib.tcr_batch_emit(ctypes.byref(self.desc), _ptr(self.structure), _ptr(self.scratch),
                                          self.scratch.numel(), _ptr(self.stage), _ptr(self.offsets), _ptr(self.row),
                                          _ptr(self.col), total, sptr), "tcr_batch_emit")
            self.stream.synchronize()
        self.total = total
        return total


def enqueue_batch(table, mode, self_search, fmt, device, stream, cap, stage_cap, local_index=True, query_ids=None,
                  ref_ids=None, lin_hint=None, lin_out=None, order_out=None, base_index=None):
    """Enqueues build, count and emit of one batch on `stream` into buffers of its own and returns a
    ``PendingBatch`` without waiting: `cap` output pairs and `stage_cap` staging words are the
    caller's estimates.  `base_index` (int64 device tensor, optional): query indices whose offsets
    are copied to pinned host memory after the count (``PendingBatch.offsets_host``), so a caller
    can slice per-cloud results with no device read of its own."""
    lib = _lib.load()
    table = np.ascontiguousarray(table)
    b = batch_desc(table, mode, self_search, local_index, query_ids, ref_ids, lin_hint, lin_out, order_out)
    s_bytes, w_bytes = _lib.batch_sizes(b)
    nq = int(table["n_query"].sum())
    cap, stage_cap = int(min(0x7fffffff, max(cap, 1))), int(min(0x7fffffff, max(stage_cap, 1)))
    sptr = ctypes.c_void_p(stream.cuda_stream)
    with torch.cuda.stream(stream):
        structure = torch.empty(max(s_bytes, 1), dtype=torch.uint8, device=device)
        scratch = torch.empty(max(w_bytes, 1), dtype=torch.uint8, device=device)
        stage = torch.empty(stage_cap, dtype=torch.int32, device=device)
        offsets = torch.empty(nq + 1, dtype=torch.int64, device=device)
        col = torch.empty(cap, dtype=torch.int64, device=device)
        row = torch.empty(cap, dtype=torch.int64, device=device) if fmt == "coo" else None
        info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
        _lib.check(lib.tcr_batch_build_structure(ctypes.byref(b), _ptr(structure), s_bytes, _ptr(scratch), w_bytes,
                                                 sptr), "tcr_batch_build_structure")
        _lib.check(lib.tcr_batch_count(ctypes.byref(b), _ptr(structure), _ptr(scratch), w_bytes, _ptr(stage),
                                       stage_cap, _ptr(offsets), None, None, ctypes.c_void_p(info.data_ptr()), sptr),
                   "tcr_batch_count")
        offsets_host = None
        if base_index is not None:
            offsets_host = torch.empty(base_index.numel(), dtype=torch.int64, pin_memory=True)
            offsets_host.copy_(offsets.index_select(0, base_index), non_blocking=True)
        _lib.check(lib.tcr_batch_emit(ctypes.byref(b), _ptr(structure), _ptr(scratch), w_bytes, _ptr(stage),
                                      _ptr(offsets), _ptr(row), _ptr(col), cap, sptr), "tcr_batch_emit")
        event = torch.cuda.Event()
        event.record(stream)
    return PendingBatch(desc=b, table=table, query_ids=query_ids, ref_ids=ref_ids, structure=structure,
                        scratch=scratch, stage=stage, offsets=offsets, col=col, row=row, info=info,
                        offsets_host=offsets_host, cap=cap, fmt=fmt, device=device, stream=stream, event=event,
                        total=None)


class BatchedAdjacency:
    """Adjacency of a batched search: one CSR (or COO) over the queries of all clouds in order,
    and per-cloud views ``adj[k]`` -- the ``SparseCSR`` / ``SparseCOO`` that ``radiusSearch``
    returns for cloud k alone, with indices inside the cloud."""

    def __init__(self, fmt, out, n_query, n_ref):
        self.format = fmt
        self.row = out["row"]
        self.col = out["col"]
        self.offsets = out["offsets"]
        self.indptr = out["indptr"]
        self.rowEntries = out["counts"]
        self.numPairs = out["total"]
        self.numRows = [int(v) for v in n_query]
        self.numCols = [int(v) for v in n_ref]
        q = np.zeros(len(self.numRows) + 1, dtype=np.int64)
        np.cumsum(self.numRows, out=q[1:])
        self.queryOffsets = q
        self._pair_off = None

    def __len__(self):
        return len(self.numRows)

    def _pairs(self):
        if self._pair_off is None:
            idx = torch.as_tensor(self.queryOffsets, device=self.offsets.device)
            self._pair_off = self.offsets.index_select(0, idx).cpu().tolist()
        return self._pair_off

    def __getitem__(self, k):
        if k < 0:
            k += len(self)
        q0, q1 = int(self.queryOffsets[k]), int(self.queryOffsets[k + 1])
        p = self._pairs()
        p0, p1 = p[k], p[k + 1]
        if self.format == "coo":
            return SparseCOO(self.row[p0:p1], self.col[p0:p1], self.numRows[k], self.numCols[k])
        indptr = (self.offsets[q0:q1 + 1] - p0).to(torch.int32)
        return SparseCSR(self.col[p0:p1], indptr, self.rowEntries[q0:q1], self.numRows[k], self.numCols[k])


def _domain_list(domain, n, dims, device):
    if domain is None or isinstance(domain, DomainDescription):
        domain = [domain] * n
    if len(domain) != n:
        raise ValueError(f"{len(domain)} domains for {n} clouds")
    out = []
    for d, dim in zip(domain, dims):
        if d is None:  # neighborhood.py:193-197: [0, 1]^d, not periodic
            out.append(([0.0] * dim, [1.0] * dim, 0))
        else:
            out.append(_domain_host(d, dim))
    return out


def radiusSearchBatch(queryPointClouds: Sequence[PointCloud],
                      referencePointClouds: Optional[Sequence[PointCloud]] = None,
                      supportOverride: Optional[float] = None, mode: str = "gather",
                      domain: Union[None, DomainDescription, Sequence[DomainDescription]] = None,
                      hashMapLength: Union[int, Sequence[int]] = 4096, format: str = "csr",
                      verbose: bool = False) -> BatchedAdjacency:
    """``radiusSearch(..., algorithm='compact')`` over many independent clouds at once.

    Cloud k searches ``queryPointClouds[k]`` against ``referencePointClouds[k]`` (itself when
    ``referencePointClouds`` is None) in ``domain[k]`` (one domain for all, a list, or None for
    the reference's default [0, 1]^d) with ``hashMapLength[k]``; clouds may differ in size,
    dimension and periodicity.  ``adj[k]`` equals what ``radiusSearch`` returns for cloud k
    alone, bit for bit.
    """
    with torch.no_grad():
        assert format in ("coo", "csr"), f"format = {format} not supported"
        assert mode in _lib.MODES, f"mode = {mode} not supported"
        n = len(queryPointClouds)
        if n == 0:
            raise ValueError("no clouds")
        self_search = referencePointClouds is None
        refs = queryPointClouds if self_search else referencePointClouds
        if len(refs) != n:
            raise ValueError(f"{n} query clouds but {len(refs)} reference clouds")
        device = _require_cuda(queryPointClouds[0].positions.device)
        dims = [pc.positions.shape[1] for pc in queryPointClouds]
        doms = _domain_list(domain, n, dims, device)
        Ls = [hashMapLength] * n if isinstance(hashMapLength, int) else list(hashMapLength)
        table = cloud_table(n)
        keep = []
        for k in range(n):
            q, r = queryPointClouds[k], refs[k]
            dim = dims[k]
            if r.positions.shape[1] != dim:
                raise ValueError(f"cloud {k}: query and reference dimensions differ")
            xq = _as_f32(q.positions, device)
            xr = xq if self_search else _as_f32(r.positions, device)
            if supportOverride is not None:
                hq = torch.full((xq.shape[0],), float(supportOverride), dtype=torch.float32, device=device)
                hr = hq if self_search else torch.full((xr.shape[0],), float(supportOverride), dtype=torch.float32,
                                                       device=device)
            else:
                hq = None if q.supports is None else _as_f32(q.supports, device)
                hr = hq if self_search else (None if r.supports is None else _as_f32(r.supports, device))
            if mode in ("gather", "symmetric", "superSymmetric") and hq is None:
                raise AssertionError(f"cloud {k}: query supports must be provided for {mode} mode")
            if mode in ("scatter", "symmetric", "superSymmetric") and hr is None:
                raise AssertionError(f"cloud {k}: reference supports must be provided for {mode} mode")
            keep.extend([xq, xr, hq, hr])
            lo, hi, mask = doms[k]
            table["dim"][k] = dim
            table["periodic_mask"][k] = mask
            table["domain_min"][k, :dim] = lo
            table["domain_max"][k, :dim] = hi
            table["hash_map_length"][k] = int(Ls[k])
            table["n_query"][k] = xq.shape[0]
            table["n_ref"][k] = xr.shape[0]
            table["query_pos"][k] = xq.data_ptr() if xq.numel() else 0
            table["ref_pos"][k] = xr.data_ptr() if xr.numel() else 0
            table["query_sup"][k] = hq.data_ptr() if hq is not None and hq.numel() else 0
            table["ref_sup"][k] = hr.data_ptr() if hr is not None and hr.numel() else 0
        if verbose:
            print(f"radiusSearchBatch: {n} clouds, {int(table['n_query'].sum())} queries, "
                  f"{int(table['n_ref'].sum())} references, mode {mode}, format {format}")
        out = run_batch(table, mode, self_search, format, device, local_index=True)
        del keep
        return BatchedAdjacency(format, out, table["n_query"], table["n_ref"])


def radius_batched(xq, xr, support, batch_x, batch_y, mode="gather", domain=None, hashMapLength=4096,
                   returnStructure=False, same_cloud=False):
    """torch_cluster-style ``radius`` with batch vectors (neighborhood.py:333-363): every batch id is
    an independent cloud (all in `domain`) and the returned (i, j) are indices into xq / xr, in
    batch-id order, then query order, then the compact walk's order -- what searching each batch id
    alone and concatenating gives.  One batched search; batch vectors need not be sorted."""
    if returnStructure:
        return _radius_per_id(xq, xr, support, batch_x, batch_y, mode, domain, hashMapLength, same_cloud)
    device = _require_cuda(xq.device)
    dim = xq.shape[1]
    if batch_x is None:
        batch_x = torch.zeros(xq.shape[0], dtype=torch.long, device=xq.device)
    if batch_y is None:
        batch_y = batch_x if same_cloud else torch.zeros(xr.shape[0], dtype=torch.long, device=xr.device)
    bx = batch_x.to(device=device, dtype=torch.long)
    by = bx if same_cloud else batch_y.to(device=device, dtype=torch.long)
    ids = torch.unique(torch.cat([bx, by]))
    C = int(ids.numel())
    if C == 0:
        e = torch.empty(0, dtype=torch.long, device=xq.device)
        return e, e
    cq = torch.searchsorted(ids, bx)
    cr = cq if same_cloud else torch.searchsorted(ids, by)
    oq = torch.argsort(cq, stable=True)
    orr = oq if same_cloud else torch.argsort(cr, stable=True)
    nq = torch.bincount(cq, minlength=C)
    nr = nq if same_cloud else torch.bincount(cr, minlength=C)
    counts = torch.stack([nq, nr]).cpu().numpy().astype(np.int64)
    xs = _as_f32(xq, device).index_select(0, oq).contiguous()
    ys = xs if same_cloud else _as_f32(xr, device).index_select(0, orr).contiguous()
    if isinstance(support, (tuple, list)):
        hq = _as_f32(support[0], device).index_select(0, oq).contiguous()
        hr = _as_f32(support[1], device).index_select(0, orr).contiguous()
    elif torch.is_tensor(support) and support.dim() > 0:
        hq = _as_f32(support, device).index_select(0, oq).contiguous()
        hr = hq if same_cloud else None
    else:
        hq = torch.full((xs.shape[0],), float(support), dtype=torch.float32, device=device)
        hr = hq if same_cloud else torch.full((ys.shape[0],), float(support), dtype=torch.float32, device=device)
    if mode in ("scatter", "symmetric", "superSymmetric") and hr is None:
        raise AssertionError(f"referenceSupports must be provided for {mode} mode")
    lo, hi, mask = _domain_list(domain, 1, [dim], device)[0]
    table = cloud_table(C)
    qoff = np.zeros(C, dtype=np.int64)
    roff = np.zeros(C, dtype=np.int64)
    np.cumsum(counts[0][:-1], out=qoff[1:])
    np.cumsum(counts[1][:-1], out=roff[1:])
    table["dim"] = dim
    table["periodic_mask"] = mask
    table["domain_min"][:, :dim] = lo
    table["domain_max"][:, :dim] = hi
    table["hash_map_length"] = int(hashMapLength)
    table["n_query"] = counts[0]
    table["n_ref"] = counts[1]
    table["query_pos"] = np.where(counts[0] > 0, xs.data_ptr() + qoff * dim * 4, 0) if xs.numel() else 0
    table["ref_pos"] = np.where(counts[1] > 0, ys.data_ptr() + roff * dim * 4, 0) if ys.numel() else 0
    if hq is not None and hq.numel():
        table["query_sup"] = np.where(counts[0] > 0, hq.data_ptr() + qoff * 4, 0)
    if hr is not None and hr.numel():
        table["ref_sup"] = np.where(counts[1] > 0, hr.data_ptr() + roff * 4, 0)
    qids = oq.to(torch.int32)
    rids = qids if same_cloud else orr.to(torch.int32)
    out = run_batch(table, mode, same_cloud, "coo", device, local_index=False, query_ids=qids, ref_ids=rids)
    i, j = out["row"], out["col"]
    if xq.device.type == "cpu":
        i, j = _to_host((i, j))
    elif xq.device.type != "cuda":
        i, j = i.to(xq.device), j.to(xq.device)
    return i, j


def _radius_per_id(xq, xr, support, batch_x, batch_y, mode, domain, hashMapLength, same_cloud):
    """``radius(..., returnStructure=True)``: one search (and one reusable structure) per batch id."""
    from .neighborhood import radiusSearch
    dev = xq.device
    if batch_x is None:
        batch_x = torch.zeros(xq.shape[0], dtype=torch.long, device=dev)
    if batch_y is None:
        batch_y = batch_x if same_cloud else torch.zeros(xr.shape[0], dtype=torch.long, device=dev)
    ids = torch.unique(torch.cat([batch_x, batch_y]))
    rows, cols, structs = [], [], {}
    for b in ids.tolist():
        qi = torch.nonzero(batch_x == b).flatten()
        ri = torch.nonzero(batch_y == b).flatten()
        if qi.numel() == 0 or ri.numel() == 0:
            continue
        if isinstance(support, (tuple, list)):
            hq, hr = support[0][qi], support[1][ri]
            fixed = None
        elif torch.is_tensor(support) and support.dim() > 0:
            hq = support[qi]
            hr = support[ri] if same_cloud else None
            fixed = None
        else:
            hq = hr = None
            fixed = float(support)
        res, structs[b] = radiusSearch(PointCloud(xq[qi], hq), PointCloud(xr[ri], hr), supportOverride=fixed,
                                       mode=mode, domain=domain, hashMapLength=hashMapLength, algorithm="compact",
                                       format="coo", returnStructure=True)
        rows.append(qi[res.row.to(qi.device)])
        cols.append(ri[res.col.to(ri.device)])
    i = torch.cat(rows) if rows else torch.empty(0, dtype=torch.long, device=dev)
    j = torch.cat(cols) if cols else torch.empty(0, dtype=torch.long, device=dev)
    return i, j, structs
