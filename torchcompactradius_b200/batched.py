"""Batched searches over many independent point clouds.

``radius_batched`` gives the torch_cluster-style ``radius(x, y, r, batch_x, batch_y)`` semantics
(reference neighborhood.py:333-363): every batch id is an independent cloud and the returned
indices are global.
"""
import torch

from .util import PointCloud


def radius_batched(xq, xr, support, batch_x, batch_y, mode="gather", domain=None, hashMapLength=4096,
                   returnStructure=False, same_cloud=False):
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
        res = radiusSearch(PointCloud(xq[qi], hq), PointCloud(xr[ri], hr), supportOverride=fixed, mode=mode,
                           domain=domain, hashMapLength=hashMapLength, algorithm="compact", format="coo",
                           returnStructure=returnStructure)
        if returnStructure:
            res, structs[b] = res
        rows.append(qi[res.row.to(qi.device)])
        cols.append(ri[res.col.to(ri.device)])
    i = torch.cat(rows) if rows else torch.empty(0, dtype=torch.long, device=dev)
    j = torch.cat(cols) if cols else torch.empty(0, dtype=torch.long, device=dev)
    if returnStructure:
        return i, j, structs
    return i, j
