"""Tuning never changes a result: every (queries per unit, blocks per SM) setting gives the same
CSR, and the autotuner leaves one of its candidates in force."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _search(x, h, dom, mode):
    import torchcompactradius_b200 as tcr
    return tcr.radiusSearch(tcr.PointCloud(x, h), mode=mode, domain=dom, algorithm="compact", format="csr")


@pytest.mark.parametrize("dim,periodic,mode", [(3, False, "symmetric"), (2, True, "gather"), (3, True, "scatter")])
def test_every_setting_gives_the_same_result(dim, periodic, mode):
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.tuning import CANDIDATES, set_tuning
    g = torch.Generator().manual_seed(dim)
    n = 30000
    x = (torch.rand(n, dim, generator=g) * 2 - 1).cuda()
    dx = 2.0 / n ** (1.0 / dim)
    h0 = (32 * dx * dx / np.pi) ** 0.5 if dim == 2 else (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)
    h = (h0 * (0.9 + 0.2 * torch.rand(n, generator=g))).cuda()
    dom = tcr.DomainDescription(torch.full((dim,), -1.0), torch.full((dim,), 1.0), torch.tensor([periodic] * dim), dim)
    from torchcompactradius_b200 import context
    with context.use(context.SearchContext()):
        set_tuning(32, 12)
        ref = _search(x, h, dom, mode)
        for cfg in CANDIDATES + [(8, 1), (16, 64)]:
            set_tuning(*cfg)
            got = _search(x, h, dom, mode)
            assert torch.equal(got.indices, ref.indices) and torch.equal(got.indptr, ref.indptr), cfg


def test_autotuner_picks_a_candidate_and_remembers_it():
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.tuning import Autotuner, set_tuning, signature
    x = (torch.rand(50000, 3) * 2 - 1).cuda()
    h = torch.full((50000,), 0.06).cuda()
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([False] * 3), 3)
    tuner = Autotuner(reps=2)
    key = signature([3], [False], 50000, "gather", 50)
    from torchcompactradius_b200 import context
    with context.use(context.SearchContext()) as ctx:
        best = tuner.tune(lambda: _search(x, h, dom, "gather"), key)
        assert best in tuner.candidates and len(tuner.timings[key]) == len(tuner.candidates)
        assert ctx.tuning() == best
        assert tuner.tune(lambda: None, key) == best  # remembered: no timing the second time


@pytest.mark.parametrize("dim,periodic,mode", [(3, False, "symmetric"), (2, True, "gather"), (3, True, "scatter"),
                                               (3, [True, False, True], "superSymmetric"), (1, True, "symmetric")])
def test_cell_scale_keeps_the_pair_set_of_points_inside_the_domain(dim, periodic, mode):
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200 import context
    from torchcompactradius_b200.tuning import same_pairs
    per = periodic if isinstance(periodic, list) else [periodic] * dim
    g = torch.Generator().manual_seed(17 + dim)
    n = 20000
    x = (torch.rand(n, dim, generator=g) * 2 - 1).cuda()
    dx = 2.0 / n ** (1.0 / dim)
    h0 = {1: 8 * dx, 2: (32 * dx * dx / np.pi) ** 0.5, 3: (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)}[dim]
    h = (h0 * (0.7 + 0.6 * torch.rand(n, generator=g))).cuda()
    dom = tcr.DomainDescription(torch.full((dim,), -1.0), torch.full((dim,), 1.0), torch.tensor(per), dim)
    with context.use(context.SearchContext()) as ctx:
        ref = _search(x, h, dom, mode)
        for m in (1.25, 1.5, 2.0, 3.0):
            ctx.cell_scale = m
            got = _search(x, h, dom, mode)
            assert torch.equal(got.indptr, ref.indptr), m
            assert same_pairs(got, ref), m


def test_autotuner_cell_scale_pick_is_remembered():
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200 import context
    from torchcompactradius_b200.tuning import CELL_SCALES, Autotuner
    x = (torch.rand(40000, 2) * 2 - 1).cuda()
    h = torch.full((40000,), 0.02).cuda()
    dom = tcr.DomainDescription(torch.full((2,), -1.0), torch.full((2,), 1.0), torch.tensor([True, True]), 2)
    tuner = Autotuner(reps=2)
    with context.use(context.SearchContext()) as ctx:
        best = tuner.tune_cell_scale(lambda: _search(x, h, dom, "gather"), key="scale-test")
        assert best in CELL_SCALES and ctx.cell_scale == best
        assert set(tuner.scale_timings["scale-test"]) == set(CELL_SCALES)  # every multiplier kept the pairs
        ctx.cell_scale = 1.0
        assert tuner.tune_cell_scale(lambda: None, key="scale-test") == best
