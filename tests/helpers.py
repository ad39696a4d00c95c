"""Shared helpers for the parity tests."""
import numpy as np
import torch

import cases


def inputs_of(c):
    """Regenerates a golden case's inputs and checks them against the stored input hash."""
    if c["kind"] == "testpy":
        q, ref, h = cases.testpy_grid(c["reduced"])
        assert cases.sha(q, ref, np.float32(h)) == c["input_sha"]
        per = [c["periodic"]] * 2
        return (q, np.full(len(q), h, np.float32), ref, np.full(len(ref), h, np.float32),
                np.array([-1, -1], np.float32), np.array([1, 1], np.float32), np.array(per))
    if c["kind"] == "cfg1":
        pos, sup = cases.cfg1_inputs()
        assert cases.sha(pos, sup) == c["input_sha"]
        return pos, sup, None, None, np.array([-1, -1], np.float32), np.array([1, 1], np.float32), np.array([True, True])
    x, hx, y, hy, dmin, dmax, per = cases.random_case(**c["params"])
    assert cases.sha(x, hx, y, hy) == c["input_sha"]
    return x, hx, y, hy, dmin, dmax, np.asarray(per)


def gpu_search(xq, hq, xr, hr, dmin, dmax, per, mode, L=4096, fmt="coo", device="cuda", **kw):
    import torchcompactradius_b200 as tcr
    t = lambda a: None if a is None else torch.as_tensor(np.asarray(a)).to(device)
    dom = tcr.DomainDescription(torch.tensor(np.asarray(dmin, np.float32)), torch.tensor(np.asarray(dmax, np.float32)),
                                torch.tensor(np.asarray(per, bool)), len(dmin))
    q = tcr.PointCloud(t(xq), t(hq))
    r = None if xr is None else tcr.PointCloud(t(xr), t(hr))
    return tcr.radiusSearch(q, r, mode=mode, domain=dom, hashMapLength=L, algorithm="compact", format=fmt, **kw)


def coo_arrays(adj):
    return adj.row.cpu().numpy(), adj.col.cpu().numpy()


def csr_rows(adj):
    indptr = adj.indptr.cpu().numpy().astype(np.int64)
    rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    return rows, adj.indices.cpu().numpy()
