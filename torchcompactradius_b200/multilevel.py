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
* every level pair's count runs first; one merged scan gives each query its CSR row; each level
  pair's emit then writes straight into its part of the row (reference level order, then the
  compact walk's order).

The pair set is therefore exactly {(i, j): dist(i, j) < thr(i, j)} under the reference's float
test -- the reference compact search's set whenever its own grid has no periodic-seam or aliasing
artefact.
"""
import ctypes
import math

import torch

from . import _lib
from .search import _check_info, _ptr, make_desc

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
    """Exact search with per-level grids; returns (row, col) for COO or (indices, indptr, rowEntries)."""
    lib = _lib.load()
    device = xq.device
    dim = xq.shape[1]
    nq, nr = xq.shape[0], xr.shape[0]
    stream = torch.cuda.current_stream(device)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    plan = plan_levels(hq, hr, mode, max_levels)
    if plan is None:
        raise ValueError("multi-level search needs finite positive supports")
    L, H = plan["L"], plan["H"]
    qlev = _levels(hq, H[0], L) if plan["use_q"] else torch.zeros(nq, dtype=torch.int64, device=device)
    rlev = _levels(hr, H[0], L) if plan["use_r"] else torch.zeros(nr, dtype=torch.int64, device=device)
    qsets = [(a, torch.nonzero(qlev == a).flatten().to(torch.int32)) for a in range(L)]
    rsets = [(b, torch.nonzero(rlev == b).flatten().to(torch.int32)) for b in range(L)]
    qsets = [(a, ids) for a, ids in qsets if ids.numel()]
    rsets = [(b, ids) for b, ids in rsets if ids.numel()]
    searches = []
    counts_total = torch.zeros(nq, dtype=torch.int64, device=device)
    for b, rids in rsets:
        yr = xr.index_select(0, rids).contiguous()
        gr = hr.index_select(0, rids).contiguous() if hr is not None else None
        for a, qids in qsets:
            Ha = H[a] if plan["use_q"] else H[0]
            Hb = H[b] if plan["use_r"] else H[0]
            if not plan["use_q"]:
                Ha = Hb
            if not plan["use_r"]:
                Hb = Ha
            T = pair_radius(mode, Ha, Hb)
            yq = xq.index_select(0, qids).contiguous()
            gq = hq.index_select(0, qids).contiguous() if hq is not None else None
            desc = make_desc(dim, mode, mask, lo, hi, 0xFFFFFFFF, yq, gq, yr, gr, False)
            desc.query_ids = qids.data_ptr()
            desc.ref_ids = rids.data_ptr()
            for k, v in enumerate(cell_sizes(T, lo, hi, mask, dim)):
                desc.hcell[k] = v
            desc.clamped_grid = 1
            s_bytes, w_bytes = _lib.search_sizes(yq.shape[0], yr.shape[0], dim)
            sbuf = torch.empty(s_bytes, dtype=torch.uint8, device=device)
            scratch = torch.empty(w_bytes, dtype=torch.uint8, device=device)
            _lib.check(lib.tcr_build_structure(ctypes.byref(desc), _ptr(sbuf), s_bytes, _ptr(scratch), w_bytes,
                                               sptr), "tcr_build_structure")
            nql = yq.shape[0]
            stage_cap = int(min(0x7fffffff, 96 * nql + 65536))
            stage = torch.empty(stage_cap, dtype=torch.int32, device=device)
            off_local = torch.empty(nql + 1, dtype=torch.int64, device=device)
            cnt_local = torch.empty(nql, dtype=torch.int64, device=device)
            info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
            _lib.check(lib.tcr_count(ctypes.byref(desc), _ptr(sbuf), _ptr(scratch), w_bytes, _ptr(stage),
                                     stage_cap, _ptr(off_local), None, _ptr(cnt_local),
                                     ctypes.c_void_p(info.data_ptr()), sptr), "tcr_count")
            counts_total.index_add_(0, qids.to(torch.int64), cnt_local)
            searches.append(dict(desc=desc, keep=(yq, gq, yr, gr, qids, rids), sbuf=sbuf, scratch=scratch,
                                 w_bytes=w_bytes, stage=stage, cnt=cnt_local, info=info))
    offsets = torch.zeros(nq + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts_total, 0, out=offsets[1:])
    total = int(offsets[-1])  # the one host synchronisation
    for s in searches:
        _check_info(s["info"])
    if fmt == "csr" and total > 0x7fffffff:
        raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
    col = torch.empty(total, dtype=torch.int64, device=device)
    row = torch.empty(total, dtype=torch.int64, device=device) if fmt == "coo" else None
    running = offsets[:-1].clone()
    for s in searches:
        qids = s["keep"][4].to(torch.int64)
        emit_off = torch.empty(qids.numel() + 1, dtype=torch.int64, device=device)
        emit_off[:-1] = running.index_select(0, qids)
        emit_off[-1] = total
        running.index_add_(0, qids, s["cnt"])
        if total:
            _lib.check(lib.tcr_emit(ctypes.byref(s["desc"]), _ptr(s["sbuf"]), _ptr(s["scratch"]), s["w_bytes"],
                                    _ptr(s["stage"]), _ptr(emit_off), _ptr(row), _ptr(col), total, sptr),
                       "tcr_emit")
        s["emit_off"] = emit_off  # keep alive until the stream passes it
    if fmt == "coo":
        return row, col
    return col, offsets.to(torch.int32), counts_total
