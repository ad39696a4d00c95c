"""Searches replayed as CUDA graphs return what the eager search returns, after input updates
and after an output that outgrew the recorded capacity."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _cloud(seed, n, dim, periodic):
    import torchcompactradius_b200 as tcr
    g = torch.Generator().manual_seed(seed)
    x = (torch.rand(n, dim, generator=g) * 2 - 1).cuda()
    dx = 2.0 / n ** (1.0 / dim)
    h0 = (32 * dx * dx / np.pi) ** 0.5 if dim == 2 else (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)
    h = (h0 * (0.9 + 0.2 * torch.rand(n, generator=g))).cuda()
    dom = tcr.DomainDescription(torch.full((dim,), -1.0), torch.full((dim,), 1.0), torch.tensor([periodic] * dim), dim)
    return x, h, dom


def _same(a, b, fmt):
    if fmt == "csr":
        assert torch.equal(a.indices, b.indices) and torch.equal(a.indptr, b.indptr)
        assert torch.equal(a.rowEntries, b.rowEntries)
    else:
        assert torch.equal(a.row, b.row) and torch.equal(a.col, b.col)


@pytest.mark.parametrize("fmt", ["csr", "coo"])
@pytest.mark.parametrize("dim,periodic,mode", [(2, True, "gather"), (3, False, "symmetric"), (3, True, "scatter")])
def test_static_search_replays_equal_eager_searches(fmt, dim, periodic, mode):
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.graphs import StaticSearch
    x, h, dom = _cloud(3, 20000, dim, periodic)
    ss = StaticSearch(tcr.PointCloud(x, h), dom, mode=mode, format=fmt)
    _same(ss.run(), tcr.radiusSearch(tcr.PointCloud(x, h), mode=mode, domain=dom, algorithm="compact", format=fmt),
          fmt)
    for step in range(3):
        x = x + 0.01 * torch.randn(x.shape, device="cuda")
        ss.update(x)
        _same(ss.run(), tcr.radiusSearch(tcr.PointCloud(x, h), mode=mode, domain=dom, algorithm="compact",
                                         format=fmt), fmt)


def test_replay_grows_the_output_when_points_crowd_together():
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.graphs import StaticSearch
    x, h, dom = _cloud(4, 8000, 3, False)
    ss = StaticSearch(tcr.PointCloud(x, h), dom, mode="gather", format="csr")
    cap0 = ss.plan.cap
    y = x * 0.5  # 8x denser: far more pairs than recorded
    ss.update(y)
    got = ss.run()
    assert ss.plan.cap > cap0
    _same(got, tcr.radiusSearch(tcr.PointCloud(y, h), mode="gather", domain=dom, algorithm="compact", format="csr"),
          "csr")
    ss.update(x)  # and back, through the newly recorded graph
    _same(ss.run(), tcr.radiusSearch(tcr.PointCloud(x, h), mode="gather", domain=dom, algorithm="compact",
                                     format="csr"), "csr")


def test_batched_plan_replays_equal_eager_batches():
    from torchcompactradius_b200 import batched
    from torchcompactradius_b200.graphs import SearchPlan
    xs, hs = [], []
    t = batched.cloud_table(5)
    for k in range(5):
        d = 2 + k % 2
        x, h, _ = _cloud(10 + k, 3000 * (k + 1), d, k % 3 == 0)
        xs.append(x)
        hs.append(h)
        t["dim"][k] = d
        t["periodic_mask"][k] = (1 << d) - 1 if k % 3 == 0 else 0
        t["domain_min"][k, :d] = -1.0
        t["domain_max"][k, :d] = 1.0
        t["n_query"][k] = t["n_ref"][k] = x.shape[0]
        t["query_pos"][k] = t["ref_pos"][k] = x.data_ptr()
        t["query_sup"][k] = t["ref_sup"][k] = h.data_ptr()
    plan = SearchPlan(t, "gather", True, "csr")
    eager = batched.run_batch(t, "gather", True, "csr", torch.device("cuda"))
    for _ in range(2):
        got = plan.replay()
        assert got["total"] == eager["total"]
        assert torch.equal(got["col"], eager["col"]) and torch.equal(got["offsets"], eager["offsets"])
