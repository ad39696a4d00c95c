"""Public search API with the reference's names, arguments and return types.

``radiusSearch`` follows src/torchCompactRadius/neighborhood.py:136-309, ``radius``
:313-363 (torch_cluster-style, batched) and ``neighborSearchExisting`` :28-129.  Every
algorithm name runs the compact-hashing CUDA path; there is no CPU fallback.
"""
from typing import Optional, Tuple, Union

import torch

from .search import CompactHashMap, _as_f32, _domain_host, _require_cuda, _to_host, compact_search
from .util import DomainDescription, PointCloud, SparseCOO, SparseCSR

ALGORITHMS = ("naive", "small", "compact", "cluster", "mlm")
MODES = ("symmetric", "scatter", "gather", "superSymmetric")


def _default_domain(dim, device):
    # neighborhood.py:193-197: [0, 1]^d, not periodic
    return DomainDescription(torch.zeros(dim, device=device), torch.ones(dim, device=device),
                             torch.zeros(dim, dtype=torch.bool, device=device), dim)


def radiusSearch(queryPointCloud: PointCloud, referencePointCloud: Optional[PointCloud] = None,
                 supportOverride: Optional[float] = None, mode: str = "gather",
                 domain: Optional[DomainDescription] = None, hashMapLength=4096, algorithm: str = "naive",
                 verbose: bool = False, format: str = "coo", returnStructure: bool = False,
                 useDenseMLM: bool = False, hashMapLengthAlgorithm: str = "primes"):
    """Fixed-radius neighbour search between two point clouds (neighborhood.py:136-309).

    Returns ``SparseCOO(row, col, numRows, numCols)`` or, with ``format='csr'``,
    ``SparseCSR(indices, indptr, rowEntries, numRows, numCols)``; with ``returnStructure`` a
    tuple ``(adjacency, CompactHashMap)``.  Row i lists the reference points j whose distance
    to query i is strictly below the mode's support: gather h_i, scatter h_j, symmetric
    (h_i + h_j)/2, superSymmetric max(h_i, h_j), periodic dimensions measured across the wrap.

    ``algorithm='compact'`` (and 'naive' / 'small', which name the same CUDA search here) returns
    the reference's compact result bit for bit.  ``algorithm='mlm'`` runs the multi-level search
    (torchcompactradius_b200.multilevel): the exact pair set of the same float test on per-level
    grids, which is the compact result wherever the compact grid itself misses nothing; 'cluster'
    needs the absent torch_cluster package, as in the reference.  ``supportOverride`` gives
    every point that support (the reference's compact path rejects it).  Outputs live on the
    queries' CUDA device (CPU inputs are searched on the current CUDA device and the result is
    returned to the CPU).
    """
    with torch.no_grad():
        assert algorithm in ("naive", "small", "compact", "mlm"), f"algorithm = {algorithm} not supported"
        assert format in ("coo", "csr"), f"format = {format} not supported"
        assert mode in MODES, f"mode = {mode} not supported"
        assert queryPointCloud is not None, "queryPointCloud is None"
        if supportOverride is not None and not isinstance(supportOverride, float):
            raise ValueError(f"supportOverride = {supportOverride} must be a float")
        qpos = queryPointCloud.positions
        dim = qpos.shape[1]
        self_cloud = referencePointCloud is None
        if self_cloud:
            referencePointCloud = queryPointCloud
        rpos = referencePointCloud.positions
        assert rpos.shape[1] == dim, f"referencePositions.shape[1] = {rpos.shape[1]} != dimensionality = {dim}"
        if domain is not None:
            assert torch.as_tensor(domain.min).shape[0] == dim, "domain.min does not match the dimensionality"
            assert torch.as_tensor(domain.max).shape[0] == dim, "domain.max does not match the dimensionality"
        if queryPointCloud.supports is not None:
            assert queryPointCloud.supports.shape[0] == qpos.shape[0], "query supports do not match the positions"
        if referencePointCloud.supports is not None:
            assert referencePointCloud.supports.shape[0] == rpos.shape[0], "reference supports do not match"
        if dim < 1 or dim > 3:
            raise RuntimeError(f"Unsupported dimension: {dim}")
        in_device = qpos.device
        device = _require_cuda(in_device)
        if domain is None:
            domain = _default_domain(dim, device)
        lo, hi, mask = _domain_host(domain, dim)
        if verbose:
            print(f"radiusSearch: {qpos.shape[0]} queries, {rpos.shape[0]} references, dim {dim}, mode {mode}, "
                  f"periodic mask {mask}, hashMapLength {hashMapLength}, format {format}")
        nq, nr = qpos.shape[0], rpos.shape[0]
        if (qpos.dtype == torch.float64 or rpos.dtype == torch.float64) and algorithm != "mlm":
            out, ds = _radius_search_f64(queryPointCloud, referencePointCloud, supportOverride, mode, domain, lo, hi,
                                         mask, hashMapLength, format, self_cloud, returnStructure, device)
            if in_device.type != "cuda":
                out = _to_host(out) if in_device.type == "cpu" else tuple(
                    None if t is None else t.to(in_device) for t in out)
            adj = SparseCOO(out[0], out[1], nq, nr) if format == "coo" else SparseCSR(out[0], out[1], out[2], nq, nr)
            return (adj, ds) if returnStructure else adj
        xq = _as_f32(qpos, device)
        same = self_cloud or (rpos.data_ptr() == qpos.data_ptr() and rpos.shape == qpos.shape
                              and rpos.stride() == qpos.stride() and rpos.dtype == qpos.dtype)
        xr = xq if same else _as_f32(rpos, device)
        if supportOverride is not None:
            hq = torch.full((nq,), supportOverride, dtype=torch.float32, device=device)
            hr = hq if same else torch.full((nr,), supportOverride, dtype=torch.float32, device=device)
        else:
            hq = None if queryPointCloud.supports is None else _as_f32(queryPointCloud.supports, device)
            hr = None if referencePointCloud.supports is None else (
                hq if (self_cloud and hq is not None) else _as_f32(referencePointCloud.supports, device))
        if mode in ("gather", "symmetric", "superSymmetric"):
            assert hq is not None, f"queryParticleSupports must be provided for {mode} mode"
        if mode in ("scatter", "symmetric", "superSymmetric"):
            assert hr is not None, f"referenceSupports must be provided for {mode} mode"
        if algorithm == "mlm":
            from .multilevel import multilevel_search
            out = multilevel_search(xq, hq, xr, hr, lo, hi, mask, mode, format)
            ds = None  # neighborhood.py:260-263: the multi-level path returns no reusable structure
        else:
            # One support h for every point: each mode's threshold is h itself (symmetric:
            # fl(h/2 + h/2) = h, superSymmetric: max(h, h) = h), so the fixed-radius search runs the
            # gather walk, whose test is d^2 - h^2 with the query's share precomputed -- the same
            # pairs with fewer operations per test than the two-support modes.
            walk_mode = "gather" if supportOverride is not None else mode
            out, ds = compact_search(xq, hq, xr, hr, lo, hi, mask, walk_mode, hashMapLength, format, same,
                                     return_structure=returnStructure, ref_pos_user=rpos,
                                     ref_sup_user=referencePointCloud.supports, fixed_support=supportOverride)
        if in_device.type != "cuda":
            out = _to_host(out) if in_device.type == "cpu" else tuple(
                None if t is None else t.to(in_device) for t in out)
        if format == "coo":
            adj = SparseCOO(out[0], out[1], nq, nr)
        else:
            adj = SparseCSR(out[0], out[1], out[2], nq, nr)
        if returnStructure:
            return adj, ds
        return adj


def _radius_search_f64(q: PointCloud, r: PointCloud, supportOverride, mode, domain, lo, hi, mask, L, fmt, self_cloud,
                       returnStructure, device):
    """Float64 positions: the reference's double search (search64.py).  Positions, supports and the
    domain must all be float64, as the reference's double operators require (their accessors raise
    otherwise)."""
    from .search64 import compact_search_f64
    need = [("positions", q.positions), ("positions", r.positions), ("domain.min", domain.min),
            ("domain.max", domain.max)]
    if supportOverride is None:
        if mode != "scatter":
            need.append(("supports", q.supports))
        if mode != "gather":
            need.append(("supports", r.supports))
    for name, t in need:
        if t is None:
            continue
        if torch.as_tensor(t).dtype != torch.float64:
            raise RuntimeError(f"expected scalar type Double but found Float ({name} of a float64 search)")
    xq = q.positions.to(device=device, dtype=torch.float64).contiguous()
    xr = xq if self_cloud else r.positions.to(device=device, dtype=torch.float64).contiguous()
    if supportOverride is not None:
        hq = torch.full((xq.shape[0],), supportOverride, dtype=torch.float64, device=device)
        hr = hq if self_cloud else torch.full((xr.shape[0],), supportOverride, dtype=torch.float64, device=device)
    else:
        hq = None if q.supports is None else q.supports.to(device=device, dtype=torch.float64).contiguous()
        hr = None if r.supports is None else (hq if self_cloud else
                                              r.supports.to(device=device, dtype=torch.float64).contiguous())
    if mode in ("gather", "symmetric", "superSymmetric"):
        assert hq is not None, f"queryParticleSupports must be provided for {mode} mode"
    if mode in ("scatter", "symmetric", "superSymmetric"):
        assert hr is not None, f"referenceSupports must be provided for {mode} mode"
    return compact_search_f64(xq, hq, xr, hr, lo, hi, mask, mode, L, fmt, self_cloud, return_structure=returnStructure,
                              ref_pos_user=r.positions, fixed_support=supportOverride)


def neighborSearchExisting(queryPointCloud: PointCloud, hashMap: CompactHashMap, mode: str = "symmetric",
                           searchRadius: int = 1, variant: str = "cpp", verbose: bool = False,
                           format: str = "coo") -> Union[SparseCOO, SparseCSR]:
    """Searches new queries against a structure returned by ``radiusSearch(...,
    returnStructure=True)`` (neighborhood.py:28-129, which fails in the reference on a
    misspelt field).  Queries are wrapped into the periodic domain as ``radiusSearch`` does, so
    the result equals ``radiusSearch`` of the same queries against the structure's cloud."""
    with torch.no_grad():
        assert mode in MODES, f"mode = {mode} not supported"
        assert format in ("coo", "csr"), f"format = {format} not supported"
        if searchRadius != 1:
            raise ValueError("only searchRadius = 1 is supported (as in the reference's compact search)")
        if not isinstance(hashMap, CompactHashMap):
            raise TypeError("hashMap must be a structure returned by this package's radiusSearch")
        dev = hashMap._device
        qpos = queryPointCloud.positions
        if qpos.shape[1] != hashMap._dim:
            raise ValueError("query dimensionality does not match the structure")
        if getattr(hashMap, "_f64", None) is not None:  # a structure of float64 references
            return _existing_f64(queryPointCloud, hashMap, mode, format, dev)
        xq = _as_f32(qpos, dev)
        sup = queryPointCloud.supports
        if sup is None and hashMap.fixedSupport is not None:
            hq = torch.full((qpos.shape[0],), float(hashMap.fixedSupport), dtype=torch.float32, device=dev)
        else:
            hq = None if sup is None else _as_f32(sup, dev)
        if mode in ("gather", "symmetric", "superSymmetric") and hq is None:
            raise ValueError(f"query supports are required for {mode} mode")
        if mode in ("scatter", "symmetric", "superSymmetric") and hashMap.referenceSupports is None \
                and hashMap.fixedSupport is None:
            raise ValueError(f"the structure has no reference supports for {mode} mode")
        xr = _as_f32(hashMap.referencePositions, dev)
        if verbose:
            print(f"neighborSearchExisting: {qpos.shape[0]} queries against {hashMap}")
        out, _ = compact_search(xq, hq, xr, None, hashMap._lo, hashMap._hi, hashMap._mask, mode,
                                hashMap.hashMapLength, format, False, structure=hashMap)
        nq, nr = qpos.shape[0], hashMap._n
        if qpos.device.type != "cuda":
            out = _to_host(out) if qpos.device.type == "cpu" else tuple(
                None if t is None else t.to(qpos.device) for t in out)
        if format == "coo":
            return SparseCOO(out[0], out[1], nq, nr)
        return SparseCSR(out[0], out[1], out[2], nq, nr)


def _existing_f64(q: PointCloud, hashMap: CompactHashMap, mode, fmt, dev):
    """neighborSearchExisting against a float64 structure: float64 queries (and supports), searched
    with the reference's double arithmetic against the structure's references."""
    from .search64 import compact_search_f64
    qpos = q.positions
    if qpos.dtype != torch.float64 or (q.supports is not None and q.supports.dtype != torch.float64):
        raise RuntimeError("expected scalar type Double but found Float (queries of a float64 structure)")
    xq = qpos.to(device=dev).contiguous()
    if q.supports is None and hashMap.fixedSupport is not None:
        hq = torch.full((xq.shape[0],), float(hashMap.fixedSupport), dtype=torch.float64, device=dev)
    else:
        hq = None if q.supports is None else q.supports.to(device=dev).contiguous()
    if mode in ("gather", "symmetric", "superSymmetric") and hq is None:
        raise ValueError(f"query supports are required for {mode} mode")
    if mode in ("scatter", "symmetric", "superSymmetric") and hashMap._f64["hr"] is None:
        raise ValueError(f"the structure has no reference supports for {mode} mode")
    out, _ = compact_search_f64(xq, hq, None, None, hashMap._lo, hashMap._hi, hashMap._mask, mode,
                                hashMap.hashMapLength, fmt, False, structure=hashMap)
    nq, nr = qpos.shape[0], hashMap._n
    if qpos.device.type != "cuda":
        out = _to_host(out) if qpos.device.type == "cpu" else tuple(
            None if t is None else t.to(qpos.device) for t in out)
    if fmt == "coo":
        return SparseCOO(out[0], out[1], nq, nr)
    return SparseCSR(out[0], out[1], out[2], nq, nr)


def radius(queryPositions: torch.Tensor, referencePositions: Optional[torch.Tensor],
           support: Union[float, torch.Tensor, Tuple[torch.Tensor, torch.Tensor]],
           batch_x: Optional[torch.Tensor] = None, batch_y: Optional[torch.Tensor] = None, mode: str = "gather",
           domain: Optional[DomainDescription] = None, hashMapLength=4096, algorithm: str = "naive",
           verbose: bool = False, returnStructure: bool = False):
    """torch_cluster-style ``radius`` (neighborhood.py:313-363, which fails in the reference).

    ``support`` is a float, a per-query tensor, or a (query, reference) tensor pair.  With
    ``batch_x``/``batch_y`` (sorted or not) every batch id is searched on its own and indices are
    global.  Returns ``(i, j)`` -- query index i, reference index j -- (plus the structures when
    ``returnStructure``)."""
    with torch.no_grad():
        yq = queryPositions
        yr = queryPositions if referencePositions is None else referencePositions

        def supports_for(nq, nr, qmask=None, rmask=None):
            if isinstance(support, float) or (torch.is_tensor(support) and support.dim() == 0):
                return None, None, float(support)
            if isinstance(support, (tuple, list)):
                hq, hr = support
            else:
                hq, hr = support, (support if referencePositions is None else None)
            if qmask is not None:
                hq = hq[qmask]
                hr = hr[rmask] if hr is not None else None
            return hq, hr, None

        if batch_x is None and batch_y is None:
            hq, hr, fixed = supports_for(yq.shape[0], yr.shape[0])
            res = radiusSearch(PointCloud(yq, hq), None if referencePositions is None else PointCloud(yr, hr),
                               supportOverride=fixed, mode=mode, domain=domain, hashMapLength=hashMapLength,
                               algorithm=algorithm, verbose=verbose, format="coo", returnStructure=returnStructure)
            if returnStructure:
                adj, ds = res
                return adj.row, adj.col, ds
            return res.row, res.col
        from .batched import radius_batched
        return radius_batched(yq, yr, support, batch_x, batch_y, mode=mode, domain=domain,
                              hashMapLength=hashMapLength, returnStructure=returnStructure,
                              same_cloud=referencePositions is None)
