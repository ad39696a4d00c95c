"""Test infrastructure: a brute-force restatement of the reference's double search (float64 inputs).

The checker for ``torchcompactradius_b200.search64`` (never imported by the product).  For
float64 positions the reference's operators run at scalar_t = double
(cppSrc/neighborhoodDynamic_cpu.cpp:504,531):
  * queries are wrapped once (util.py:375-387) and references twice (that, then
    compactHashing/cppSearch.py:221): remainder(x - min, max - min) + min on periodic dimensions,
    with torch's own remainder;
  * per pair, common.h:106-129: diff = moduloOp(x_i, x_j, max - min) =
    ((x_i - x_j + h/2) - floor((x_i - x_j + h/2) / h) * h) - h/2 on periodic dimensions, x_i - x_j
    otherwise; sum += diff * diff; dist = sqrt(sum);
  * neighborhoodDynamic.h:59-70: dist < h_i (gather), h_j (scatter), (h_i + h_j) / 2 (symmetric),
    max(h_i, h_j) (superSymmetric), all in double.
This is the pair set of the reference's compact search wherever its grid has at least 3 cells on
every periodic dimension (with fewer it reports some pairs twice) and every candidate lies in a
query's stencil, which its cell size (never below the largest support) guarantees.  It is pinned to
the reference's own outputs by tests/golden/f64_cases.npz (tests/test_oracle.py).
"""
import numpy as np


def wrap(x, lo, hi, periodic):
    import torch
    t = torch.as_tensor(np.asarray(x, np.float64))
    cols = []
    for d in range(t.shape[1]):
        if periodic[d]:
            cols.append(torch.remainder(t[:, d] - float(lo[d]), float(hi[d]) - float(lo[d])) + float(lo[d]))
        else:
            cols.append(t[:, d])
    return torch.stack(cols, 1).numpy()


def radius_search(xq, hq, xr, hr, lo, hi, periodic, mode):
    """Returns (row, col) int64 in row-major order (cols ascending within a row)."""
    self_search = xr is None
    xq = np.asarray(xq, np.float64)
    xr = xq if self_search else np.asarray(xr, np.float64)
    hq = None if hq is None else np.asarray(hq, np.float64)
    hr = hq if self_search else (None if hr is None else np.asarray(hr, np.float64))
    q = wrap(xq, lo, hi, periodic)
    r = wrap(wrap(xr, lo, hi, periodic), lo, hi, periodic)
    ext = np.asarray(hi, np.float64) - np.asarray(lo, np.float64)
    rows, cols = [], []
    for i in range(q.shape[0]):
        s = np.zeros(r.shape[0], np.float64)
        for d in range(q.shape[1]):
            if periodic[d]:
                h = ext[d]
                t = (q[i, d] - r[:, d]) + h / 2.0
                diff = (t - np.floor(t / h) * h) - h / 2.0
            else:
                diff = q[i, d] - r[:, d]
            s = s + diff * diff
        dist = np.sqrt(s)
        if mode == "gather":
            thr = np.full(r.shape[0], hq[i])
        elif mode == "scatter":
            thr = hr
        elif mode == "symmetric":
            thr = (hq[i] + hr) / 2.0
        else:
            thr = np.where(hq[i] < hr, hr, hq[i])
        j = np.nonzero(dist < thr)[0]
        rows.append(np.full(j.shape[0], i, np.int64))
        cols.append(j.astype(np.int64))
    if not rows:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(rows), np.concatenate(cols)
