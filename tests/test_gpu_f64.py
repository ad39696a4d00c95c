"""Parity of the float64 search with the reference's own double search."""
import numpy as np
import pytest
import torch

import cases
import f64_fixtures as fx
from oracle import search64

pytestmark = pytest.mark.gpu

CASES = fx.load()


def run(x, hx, y, hy, lo, hi, per, mode, fmt, device="cuda"):
    import torchcompactradius_b200 as tcr
    t = lambda a: None if a is None else torch.as_tensor(np.asarray(a, np.float64)).to(device)
    dom = tcr.DomainDescription(t(lo), t(hi), torch.as_tensor(np.asarray(per, bool)), len(lo))
    q = tcr.PointCloud(t(x), t(hx))
    r = None if y is None else tcr.PointCloud(t(y), t(hy))
    return tcr.radiusSearch(q, r, mode=mode, domain=dom, algorithm="compact", format=fmt)


@pytest.mark.parametrize("case", CASES, ids=[fx.name(c) for c in CASES])
def test_reference_double_search_fixtures(case):
    x, hx, y, hy, lo, hi, per = fx.inputs(case)
    coo = run(x, hx, y, hy, lo, hi, per, case["mode"], "coo")
    assert coo.row.numel() == case["pairs"]
    assert cases.pair_sha(coo.row.cpu().numpy(), coo.col.cpu().numpy()) == case["pair_sha"]
    csr = run(x, hx, y, hy, lo, hi, per, case["mode"], "csr")
    assert np.array_equal(csr.rowEntries.cpu().numpy().astype(np.int32), case["row_counts"])
    indptr = csr.indptr.cpu().numpy().astype(np.int64)
    assert indptr[0] == 0 and np.array_equal(np.diff(indptr), case["row_counts"])
    assert torch.equal(csr.indices.cpu(), coo.col.cpu())  # same row-major order in both formats


@pytest.mark.parametrize("mode", ["gather", "symmetric"])
def test_larger_periodic_cloud_against_the_oracle(mode):
    import f64_cases
    x, hx, _, _, lo, hi, per = f64_cases.f64_case(7, 3, 8000, 0, 50, [True, True, False])
    coo = run(x, hx, None, None, lo, hi, per, mode, "coo")
    row, col = search64.radius_search(x, hx, None, None, lo, hi, per, mode)
    assert coo.row.numel() == row.size
    assert cases.pair_sha(coo.row.cpu().numpy(), coo.col.cpu().numpy()) == cases.pair_sha(row, col)


def test_cpu_inputs_and_mismatched_dtypes():
    import torchcompactradius_b200 as tcr
    c = CASES[0]
    x, hx, y, hy, lo, hi, per = fx.inputs(c)
    coo = run(x, hx, y, hy, lo, hi, per, c["mode"], "coo", device="cpu")
    assert coo.row.device.type == "cpu" and coo.row.numel() == c["pairs"]
    dom32 = tcr.DomainDescription(torch.tensor(lo, dtype=torch.float32), torch.tensor(hi, dtype=torch.float32),
                                  torch.as_tensor(per), len(lo))
    with pytest.raises(RuntimeError):  # the reference's double operators reject a float32 domain
        tcr.radiusSearch(tcr.PointCloud(torch.tensor(x).cuda(), torch.tensor(hx).cuda()), None, mode=c["mode"],
                         domain=dom32, algorithm="compact")



@pytest.mark.parametrize("mode", ["gather", "symmetric"])
def test_returned_structure_serves_new_float64_queries(mode):
    """returnStructure with float64 inputs, then neighborSearchExisting with other float64 queries:
    the same pairs as radiusSearch of those queries against the structure's references."""
    import f64_cases
    import torchcompactradius_b200 as tcr
    x, hx, y, hy, lo, hi, per = f64_cases.f64_case(21, 3, 3000, 2000, 40, [True, False, True])
    hy = hy * 0.9  # the structure's cells were sized for the references' supports
    t = lambda a: torch.as_tensor(a).cuda()
    dom = tcr.DomainDescription(t(lo), t(hi), torch.as_tensor(per), 3)
    adj, ds = tcr.radiusSearch(tcr.PointCloud(t(x), t(hx)), None, mode=mode, domain=dom, algorithm="compact",
                               returnStructure=True)
    again = tcr.neighborSearchExisting(tcr.PointCloud(t(y), t(hy)), ds, mode=mode)
    direct = tcr.radiusSearch(tcr.PointCloud(t(y), t(hy)), tcr.PointCloud(t(x), t(hx)), mode=mode, domain=dom,
                              algorithm="compact")
    assert again.row.numel() == direct.row.numel()
    assert cases.pair_sha(again.row.cpu().numpy(), again.col.cpu().numpy()) == \
        cases.pair_sha(direct.row.cpu().numpy(), direct.col.cpu().numpy())
    row, col = search64.radius_search(y, hy, x, hx, lo, hi, per, mode)
    assert cases.pair_sha(row, col) == cases.pair_sha(direct.row.cpu().numpy(), direct.col.cpu().numpy())
