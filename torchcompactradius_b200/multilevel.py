"""Multi-level cells for widely varying supports (``radiusSearch(..., algorithm='mlm')``).

The reference's multi-level memory search (src/torchCompactRadius/multiLevelMemory/wrapper.py:
145-308) assigns each point a level l with cell size hCell * 2^l and searches 3^d cells at the
query's level (cppSrc/multiLevelMemory/mlmUtil.h:246).  It loses pairs (its Morton levels are
shifted for 2D in 3D, C '%' wraps negative cells, and it takes queries from the reference set).
This module keeps the idea and makes it exact:

* supports define L nested levels H_l = H_top / 2^(L-1-l), H_top = max support * (1 + 1e-3);
  a point belongs to the smallest level whose H_l covers its support (with that margin);
* for every (query level a, reference level b) present, the queries of level a are searched
  against the references of level b on a grid whose cells cover the largest threshold such a pair
  can have -- gather H_a, scatter H_b, symmetric (H_a + H_b)/2, superSymmetric max(H_a, H_b) --
  with the CUDA compact kernels in clamped-grid mode (exact for any input);
* all level pairs run as the clouds of one batched search: one count, one merged scan that gives
  each query its CSR row, and one emit that writes every level pair straight into its part of
  the row (reference level order, then the compact walk's order).

The pair set is therefore exactly {(i, j): dist(i, j) < thr(i, j)} under the reference's float
test -- the reference compact search's set whenever its own grid has no periodic-seam or aliasing
artefact.
"""
import ctypes
import math

import torch

from . import _lib
from . import context as _context
from .search import _check_info, _ptr

GROW = 1.0 + 1e-3  # covers cell-index rounding and the seam cell's width error


def _levels(h, H0, L):
    """Smallest level l with h * GROW <= H0 * 2^l (clamped into [0, L-1])."""
    lv = torch.ceil(torch.log2(torch.clamp(h.double() * GROW / H0, min=1e-300)) - 1e-12)
    return torch.clamp(lv, 0, L - 1).to(torch.int64)


def plan_levels(hq, hr, mode, max_levels=4):
    use_q = mode in ("gather", "symmetric", "superSymmetric")
    use_r = mode in ("scatter", "symmetric", "superSymmetric")
    parts = [t for t, u in ((hq, use_q), (hr, use_r)) if u and t is not None and t.numel()]
    if not parts:
        return None
    hs = torch.cat(parts)
    hmax = float(hs.max())
    hmin = float(hs.min())
    if not (math.isfinite(hmax) and hmax > 0):
        return None
    L = 1
    if hmin > 0 and math.isfinite(hmin):
        L = int(min(max_levels, max(1, math.ceil(math.log2(hmax / hmin)) + 1)))
    H_top = hmax * GROW
    H = [H_top / 2 ** (L - 1 - l) for l in range(L)]
    return dict(L=L, H=H, use_q=use_q, use_r=use_r)


def pair_radius(mode, Ha, Hb):
    if mode == "gather":
        return Ha
    if mode == "scatter":
        return Hb
    if mode == "symmetric":
        return 0.5 * (Ha + Hb)
    return max(Ha, Hb)


def cell_sizes(T, lo, hi, mask, dim):
    """Per-dimension cells >= T; on periodic dims a whole number of cells spans the domain."""
    out = []
    for d in range(dim):
        if (mask >> d) & 1:
            ext = float(hi[d]) - float(lo[d])
            n = max(1, int(math.floor(ext / T)))
            out.append(ext / n)
        else:
            out.append(T)
    return out


def multilevel_search(xq, hq, xr, hr, lo, hi, mask, mode, fmt, max_levels=4):
    """Exact search with per-level grids; returns (row, col) for COO or (indices, indptr, rowEntries).

    Every (query level, reference level) pair is one cloud of a single batched search (its query
    and reference subsets, its own cell sizes, the clamped-grid semantics), so the whole search is
    one build, one count and one emit.  The counts of a query's level pairs are summed into its CSR
    row; each level pair's emit then writes into its part of the row (reference level order, then
    the compact walk's order) through the emit's per-query start offsets."""
    import numpy as np

    from .batched import batch_desc, cloud_table
    lib = _lib.load()
    device = xq.device
    dim = xq.shape[1]
    nq = xq.shape[0]
    stream = torch.cuda.current_stream(device)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    plan = plan_levels(hq, hr, mode, max_levels)
    if plan is None:
        raise ValueError("multi-level search needs finite positive supports")
    L, H = plan["L"], plan["H"]
    qlev = _levels(hq, H[0], L) if plan["use_q"] else torch.zeros(nq, dtype=torch.int64, device=device)
    rlev = _levels(hr, H[0], L) if plan["use_r"] else torch.zeros(xr.shape[0], dtype=torch.int64, device=device)
    qsets, rsets = [], []
    for a in range(L):
        ids = torch.nonzero(qlev == a).flatten().to(torch.int32)
        if ids.numel():
            qsets.append((a, ids, xq.index_select(0, ids).contiguous(),
                          hq.index_select(0, ids).contiguous() if hq is not None else None))
    for b in range(L):
        ids = torch.nonzero(rlev == b).flatten().to(torch.int32)
        if ids.numel():
            rsets.append((b, ids, xr.index_select(0, ids).contiguous(),
                          hr.index_select(0, ids).contiguous() if hr is not None else None))
    pairs = [(q, r) for r in rsets for q in qsets]  # reference level major: the order within a row
    total = 0
    counts_total = torch.zeros(nq, dtype=torch.int64, device=device)
    if pairs:
        table = cloud_table(len(pairs))
        for k, ((a, qids, yq, gq), (b, rids, yr, gr)) in enumerate(pairs):
            Ha = H[a] if plan["use_q"] else H[0]
            Hb = H[b] if plan["use_r"] else H[0]
            if not plan["use_q"]:
                Ha = Hb
            if not plan["use_r"]:
                Hb = Ha
            table["dim"][k] = dim
            table["periodic_mask"][k] = mask
            table["domain_min"][k, :dim] = lo
            table["domain_max"][k, :dim] = hi
            table["hash_map_length"][k] = 0xFFFFFFFF
            table["n_query"][k] = yq.shape[0]
            table["n_ref"][k] = yr.shape[0]
            table["query_pos"][k] = yq.data_ptr()
            table["ref_pos"][k] = yr.data_ptr()
            table["query_sup"][k] = gq.data_ptr() if gq is not None else 0
            table["ref_sup"][k] = gr.data_ptr() if gr is not None else 0
            table["hcell"][k, :dim] = cell_sizes(pair_radius(mode, Ha, Hb), lo, hi, mask, dim)
            table["clamped_grid"][k] = 1
        qids_all = torch.cat([q[1] for q, r in pairs])
        rids_all = torch.cat([r[1] for q, r in pairs])
        desc = batch_desc(table, mode, False, local_index=False, query_ids=qids_all, ref_ids=rids_all)
        s_bytes, w_bytes = _lib.batch_sizes(desc)
        nqb = int(table["n_query"].sum())
        sbuf = torch.empty(s_bytes, dtype=torch.uint8, device=device)
        scratch = torch.empty(w_bytes, dtype=torch.uint8, device=device)
        ctx = _context.current()
        stage_cap = int(min(0x7fffffff, ctx.level_stage_per_query * 1.1 * nqb + 65536))
        stage = torch.empty(stage_cap, dtype=torch.int32, device=device)
        off_b = torch.empty(nqb + 1, dtype=torch.int64, device=device)
        cnt_b = torch.empty(nqb, dtype=torch.int64, device=device)
        info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
        _lib.check(lib.tcr_batch_build_structure(ctypes.byref(desc), _ptr(sbuf), s_bytes, _ptr(scratch), w_bytes,
                                                 sptr), "tcr_batch_build_structure")
        _lib.check(lib.tcr_batch_count(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage), stage_cap,
                                       _ptr(off_b), None, _ptr(cnt_b), ctypes.c_void_p(info.data_ptr()), sptr),
                   "tcr_batch_count")
        counts_total.index_add_(0, qids_all.long(), cnt_b)
    offsets = torch.zeros(nq + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts_total, 0, out=offsets[1:])
    total = int(offsets[-1])  # the one host synchronisation
    if pairs:
        _check_info(info)
        ctx.level_stage_per_query = max(int(info[4]) / max(nqb, 1), 1.0)
    if fmt == "csr" and total > 0x7fffffff:
        raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
    col = torch.empty(total, dtype=torch.int64, device=device)
    row = torch.empty(total, dtype=torch.int64, device=device) if fmt == "coo" else None
    if pairs and total:
        # each level pair's queries start after the query's earlier reference levels
        emit_off = torch.empty(nqb + 1, dtype=torch.int64, device=device)
        running = offsets[:-1].clone()
        base = 0
        for q, r in pairs:
            qids = q[1].long()
            m = qids.numel()
            emit_off[base:base + m] = running.index_select(0, qids)
            running.index_add_(0, qids, cnt_b[base:base + m])
            base += m
        emit_off[-1] = total
        _lib.check(lib.tcr_batch_emit(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage),
                                      _ptr(emit_off), _ptr(row), _ptr(col), total, sptr), "tcr_batch_emit")
    if fmt == "coo":
        return row, col
    return col, offsets.to(torch.int32), counts_total
