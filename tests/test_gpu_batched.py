"""Batched searches: every cloud of a batch gets exactly what it gets searched alone.

The single-cloud compact search is pinned to the reference by the other parity tests; here each
cloud's slice of one batched search (one set of launches over all clouds) must equal the single
search of that cloud element for element -- CSR indices, indptr and rowEntries, COO rows and
columns, in the same order -- and a few clouds are also checked against the CPU oracle.
"""
import numpy as np
import pytest
import torch

import cases
from helpers import gpu_search

pytestmark = pytest.mark.gpu

MODES = ("gather", "scatter", "symmetric", "superSymmetric")


def _clouds(seed, n_clouds, dims=(2, 3), sizes=(0, 2000), self_search=True, periodic_any=True):
    """Uneven random clouds: per cloud a dimension, a size (log-uniform, some empty or tiny), a
    box, a periodicity and supports for about 20-40 neighbours."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_clouds):
        dim = int(rng.choice(dims))
        n = int(np.exp(rng.uniform(np.log(max(sizes[0], 1)), np.log(sizes[1])))) if sizes[1] > 1 else 0
        if k % 9 == 4:
            n = 0  # empty cloud
        if k % 11 == 6:
            n = 3  # tiny cloud
        ext = rng.uniform(1.0, 3.0, dim).astype(np.float32)
        per = rng.random(dim) < 0.5 if periodic_any else np.zeros(dim, bool)
        vol = float(np.prod(ext))
        target = 30.0 if dim == 2 else 40.0
        dens = max(n, 1) / vol
        h = (target / (np.pi * dens)) ** 0.5 if dim == 2 else (3 * target / (4 * np.pi * dens)) ** (1 / 3)
        h = float(min(h, 0.3 * ext.min()))
        lo = rng.uniform(-1.0, 0.0, dim).astype(np.float32)
        x = (lo + rng.random((n, dim)) * ext).astype(np.float32)
        hx = (h * rng.uniform(0.9, 1.1, n)).astype(np.float32)
        if self_search:
            y, hy = None, None
        else:
            m = max(0, int(n * rng.uniform(0.5, 1.5)))
            y = (lo + rng.random((m, dim)) * ext).astype(np.float32)
            hy = (h * rng.uniform(0.9, 1.1, m)).astype(np.float32)
        L = int(rng.choice([4096, 97, 1 << 20]))
        out.append(dict(x=x, hx=hx, y=y, hy=hy, lo=lo, hi=(lo + ext).astype(np.float32), per=per, L=L))
    return out


def _dom(c):
    import torchcompactradius_b200 as tcr
    return tcr.DomainDescription(torch.tensor(c["lo"]), torch.tensor(c["hi"]), torch.tensor(c["per"]), len(c["lo"]))


def _batch(clouds, mode, fmt):
    import torchcompactradius_b200 as tcr
    t = lambda a: None if a is None else torch.as_tensor(a).cuda()
    q = [tcr.PointCloud(t(c["x"]), t(c["hx"])) for c in clouds]
    self_search = clouds[0]["y"] is None
    r = None if self_search else [tcr.PointCloud(t(c["y"]), t(c["hy"])) for c in clouds]
    return tcr.radiusSearchBatch(q, r, mode=mode, domain=[_dom(c) for c in clouds],
                                 hashMapLength=[c["L"] for c in clouds], format=fmt)


def _single(c, mode, fmt):
    return gpu_search(c["x"], c["hx"], c["y"], c["hy"], c["lo"], c["hi"], c["per"], mode, c["L"], fmt)


def _same(a, b, fmt):
    if fmt == "csr":
        assert torch.equal(a.indices, b.indices)
        assert torch.equal(a.indptr, b.indptr)
        assert torch.equal(a.rowEntries, b.rowEntries)
    else:
        assert torch.equal(a.row, b.row)
        assert torch.equal(a.col, b.col)
    assert a.numRows == b.numRows and a.numCols == b.numCols


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("fmt", ["csr", "coo"])
def test_batch_equals_single_searches_mixed_dims_self(mode, fmt):
    clouds = _clouds(10 + MODES.index(mode), 24)
    adj = _batch(clouds, mode, fmt)
    assert len(adj) == len(clouds)
    total = 0
    for k, c in enumerate(clouds):
        if c["x"].shape[0] == 0:
            assert adj[k].numRows == 0
            continue
        _same(adj[k], _single(c, mode, fmt), fmt)
        total += adj[k].col.numel() if fmt == "coo" else adj[k].indices.numel()
    assert total == adj.numPairs and total > 0


@pytest.mark.parametrize("mode", MODES)
def test_batch_equals_single_searches_distinct_clouds(mode):
    clouds = _clouds(30 + MODES.index(mode), 16, self_search=False)
    adj = _batch(clouds, mode, "csr")
    for k, c in enumerate(clouds):
        if c["x"].shape[0] == 0:
            continue
        if c["y"].shape[0] == 0 and mode != "gather":
            continue  # no reference supports to size the grid from: the single search rejects it too
        _same(adj[k], _single(c, mode, "csr"), "csr")


@pytest.mark.parametrize("dims", [(1,), (2,), (3,)])
def test_batch_of_one_class(dims):
    clouds = _clouds(50 + dims[0], 12, dims=dims, sizes=(100, 3000))
    adj = _batch(clouds, "symmetric", "csr")
    for k, c in enumerate(clouds):
        if c["x"].shape[0]:
            _same(adj[k], _single(c, "symmetric", "csr"), "csr")


def test_batch_clouds_match_the_oracle():
    from oracle import compact
    clouds = _clouds(77, 10, sizes=(200, 1500))
    adj = _batch(clouds, "gather", "coo")
    for k, c in enumerate(clouds):
        if c["x"].shape[0] == 0:
            continue
        o = compact.radius_search(c["x"], c["hx"], None, None, c["lo"], c["hi"], c["per"], "gather", c["L"])
        got = cases.canonical(adj[k].row.cpu().numpy(), adj[k].col.cpu().numpy())
        want = cases.canonical(o.row, o.col)
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(adj[k].row.cpu().numpy(), o.row)


def test_batch_many_small_clouds():
    clouds = _clouds(91, 300, sizes=(1, 200))
    adj = _batch(clouds, "gather", "csr")
    for k in (0, 1, 57, 150, 299):
        c = clouds[k]
        if c["x"].shape[0]:
            _same(adj[k], _single(c, "gather", "csr"), "csr")


def test_radius_with_batch_vectors_matches_per_id_searches():
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.batched import _radius_per_id
    rng = np.random.default_rng(5)
    n = 20000
    x = torch.tensor(rng.random((n, 3)).astype(np.float32), device="cuda")
    bx = torch.tensor(rng.integers(0, 7, n), device="cuda")  # unsorted batch ids
    h = torch.full((n,), 0.08, device="cuda")
    i, j = tcr.radius(x, None, h, bx, None, mode="gather")
    i0, j0, _ = _radius_per_id(x, x, h, bx, bx, "gather", None, 4096, True)
    assert torch.equal(i, i0) and torch.equal(j, j0)
    y = torch.tensor(rng.random((15000, 3)).astype(np.float32), device="cuda")
    by = torch.tensor(rng.integers(1, 9, 15000), device="cuda")
    i, j = tcr.radius(x, y, 0.07, bx, by, mode="gather")
    i0, j0, _ = _radius_per_id(x, y, 0.07, bx, by, "gather", None, 4096, False)
    assert torch.equal(i, i0) and torch.equal(j, j0)
    assert bool((bx[i] == by[j]).all())


def test_batch_reports_a_cloud_without_grid():
    import torchcompactradius_b200 as tcr
    clouds = _clouds(3, 4, dims=(2,), sizes=(100, 500))
    clouds[2]["hx"][:] = 100.0  # support larger than the domain: no grid
    with pytest.raises(ValueError, match="1 cloud"):
        _batch(clouds, "gather", "csr")
