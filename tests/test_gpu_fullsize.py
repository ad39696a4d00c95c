"""Full-size workloads against the C oracle.

The benchmark's adaptive-resolution workload (2^22 points, 70% in Gaussian blobs, supports with a
ratio up to 4, periodic in x, scatter, COO) is searched in full on the device by the single-level
compact search -- whose blob-core work units have thousands of candidates each -- and by the
multi-level search; the rows of the first 65,536 queries are compared with the oracle's search of
those queries against all 2^22 points.  Every cloud of the benchmark's 256-cloud batched workload
is compared with the oracle by its canonical pair set.  supportOverride and radius() with batch
vectors are checked against the oracle on uniform supports.
"""
import hashlib
import os
import sys

import numpy as np
import pytest
import torch

from oracle import compact

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def _pair_digest(row, col, ncols):
    """SHA-256 of the pairs sorted by (row, col), through one int64 key per pair."""
    key = np.asarray(row, np.int64) * np.int64(max(int(ncols), 1)) + np.asarray(col, np.int64)
    key.sort()
    return hashlib.sha256(key.tobytes()).hexdigest(), len(key)


def _rows_below(adj_row, adj_col, nsub):
    r = adj_row
    keep = r < nsub
    return r[keep].cpu().numpy(), adj_col[keep].cpu().numpy()


@pytest.mark.slow
@pytest.mark.parametrize("algorithm", ["compact", "mlm"])
def test_adaptive_2e22_first_queries_match_the_oracle(algorithm):
    import bench
    import torchcompactradius_b200 as tcr
    x, h = bench.make_adaptive_workload()
    n, nsub = x.shape[0], 65536
    lo, hi, per = np.full(3, -1.0, np.float32), np.full(3, 1.0, np.float32), np.array([True, False, False])
    dom = tcr.DomainDescription(torch.tensor(lo), torch.tensor(hi), torch.tensor(per), 3)
    xd, hd = x.cuda(), h.cuda()
    adj = tcr.radiusSearch(tcr.PointCloud(xd, hd), mode="scatter", domain=dom, hashMapLength=4096,
                           algorithm=algorithm, format="coo")
    row, col = _rows_below(adj.row, adj.col, nsub)
    del adj
    xn, hn = x.numpy(), h.numpy()
    o = compact.radius_search(xn[:nsub], hn[:nsub], xn, hn, lo, hi, per, "scatter", 4096)
    np.testing.assert_array_equal(np.bincount(row, minlength=nsub), o.counts)
    assert _pair_digest(row, col, n) == _pair_digest(o.row, o.col, n)


@pytest.mark.slow
def test_batched_256_clouds_each_match_the_oracle():
    import bench
    from torchcompactradius_b200 import batched
    clouds = bench.make_batched_workload()
    C = len(clouds)
    table = batched.cloud_table(C)
    keep = []
    for k, c in enumerate(clouds):
        d, n = c["dim"], c["x"].shape[0]
        x, hx = c["x"].cuda(), c["h"].cuda()
        keep += [x, hx]
        table["dim"][k] = d
        table["periodic_mask"][k] = sum(1 << i for i, p in enumerate(c["periodic"]) if p)
        table["domain_min"][k, :d] = -1.0
        table["domain_max"][k, :d] = 1.0
        table["hash_map_length"][k] = 4096
        table["n_query"][k] = table["n_ref"][k] = n
        table["query_pos"][k] = table["ref_pos"][k] = x.data_ptr()
        table["query_sup"][k] = table["ref_sup"][k] = hx.data_ptr()
    out = batched.run_batch(table, "gather", True, "csr", torch.device("cuda"), local_index=True)
    offsets = out["offsets"].cpu().numpy()
    col_all = out["col"]
    q0 = 0
    total = 0
    for k, c in enumerate(clouds):
        n = c["x"].shape[0]
        p0, p1 = int(offsets[q0]), int(offsets[q0 + n])
        counts = np.diff(offsets[q0:q0 + n + 1])
        row = np.repeat(np.arange(n, dtype=np.int64), counts)
        col = col_all[p0:p1].cpu().numpy()
        d = c["dim"]
        o = compact.radius_search(c["x"].numpy(), c["h"].numpy(), None, None, np.full(d, -1.0, np.float32),
                                  np.full(d, 1.0, np.float32), np.array(c["periodic"]), "gather", 4096)
        np.testing.assert_array_equal(counts, o.counts, err_msg=f"cloud {k}")
        assert _pair_digest(row, col, n) == _pair_digest(o.row, o.col, n), f"cloud {k}"
        total += p1 - p0
        q0 += n
    assert total == out["total"]


@pytest.mark.parametrize("mode", ["gather", "scatter", "symmetric", "superSymmetric"])
@pytest.mark.parametrize("dim,per", [(2, [True, False]), (3, [False, False, False]), (3, [True, True, True])])
def test_support_override_matches_the_oracle(mode, dim, per):
    import torchcompactradius_b200 as tcr
    rng = np.random.default_rng(11 + dim)
    n = 60000
    x = (rng.random((n, dim)) * 2 - 1).astype(np.float32)
    h = np.float32(0.03 if dim == 2 else 0.06)
    lo, hi = np.full(dim, -1.0, np.float32), np.full(dim, 1.0, np.float32)
    dom = tcr.DomainDescription(torch.tensor(lo), torch.tensor(hi), torch.tensor(per), dim)
    adj = tcr.radiusSearch(tcr.PointCloud(torch.tensor(x).cuda(), None), supportOverride=float(h), mode=mode,
                           domain=dom, algorithm="compact", format="coo")
    hs = np.full(n, h, np.float32)
    o = compact.radius_search(x, hs, None, None, lo, hi, np.array(per), mode, 4096)
    assert _pair_digest(adj.row.cpu().numpy(), adj.col.cpu().numpy(), n) == _pair_digest(o.row, o.col, n)


def test_radius_with_batch_vectors_matches_the_oracle():
    import torchcompactradius_b200 as tcr
    rng = np.random.default_rng(21)
    nx, ny, r = 30000, 20000, 0.06
    x = rng.random((nx, 3)).astype(np.float32)
    y = rng.random((ny, 3)).astype(np.float32)
    bx = rng.integers(0, 6, nx)
    by = rng.integers(1, 8, ny)
    i, j = tcr.radius(torch.tensor(x).cuda(), torch.tensor(y).cuda(), r, torch.tensor(bx).cuda(),
                      torch.tensor(by).cuda(), mode="gather")
    i, j = i.cpu().numpy(), j.cpu().numpy()
    lo, hi, per = np.zeros(3, np.float32), np.ones(3, np.float32), np.zeros(3, bool)
    want_i, want_j = [], []
    for b in sorted(set(bx.tolist()) & set(by.tolist())):
        qi, rj = np.nonzero(bx == b)[0], np.nonzero(by == b)[0]
        o = compact.radius_search(x[qi], np.full(len(qi), r, np.float32), y[rj], np.full(len(rj), r, np.float32),
                                  lo, hi, per, "gather", 4096)
        want_i.append(qi[o.row])
        want_j.append(rj[o.col])
    want_i, want_j = np.concatenate(want_i), np.concatenate(want_j)
    assert _pair_digest(i, j, ny) == _pair_digest(want_i, want_j, ny)
    assert len(i) > 0 and bool((bx[i] == by[j]).all())
