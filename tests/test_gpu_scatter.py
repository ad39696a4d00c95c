"""Parity of the device scatter operators with the reference's outputs and with the oracle."""
import numpy as np
import pytest
import torch

import scatter_fixtures as fx
from oracle import scatter as oracle_scatter

pytestmark = pytest.mark.gpu

CASES = fx.load()
REDUCES = ["sum", "mean", "mul", "min", "max"]


def tcr():
    import torchcompactradius_b200 as m
    return m


def run(src, index, dim, reduce, out=None, dim_size=None):
    fn = getattr(tcr(), "scatter_" + reduce)
    res = fn(src, index, dim, out, dim_size)
    return res if reduce in ("min", "max") else (res, None)


def oracle(src_t, index_t, dim, reduce, out_t=None, dim_size=None):
    from torchcompactradius_b200.scatter import broadcast
    bf16 = src_t.dtype == torch.bfloat16
    src = src_t.float().cpu().numpy() if bf16 else src_t.cpu().numpy()
    d = dim + src_t.dim() if dim < 0 else dim
    index_b = broadcast(index_t.cpu(), src_t.cpu(), d).numpy()
    out = None
    if out_t is not None:
        out = out_t.float().cpu().numpy() if bf16 else out_t.cpu().numpy()
    res, arg = oracle_scatter.scatter(src, index_b, dim, reduce, out=out, dim_size=dim_size, bf16=bf16)
    dt = "bfloat16" if bf16 else None
    return fx.bits_of_numpy(res, dt), arg


def check_bits(got, want_bits, dtype):
    assert fx.same_bits(fx.bits_of_torch(got), want_bits, "bfloat16" if dtype == torch.bfloat16 else str(dtype))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_fixtures_bit_exact(case):
    dt = case["dtype"]
    src = fx.to_torch(case["src"], dt).cuda()
    index = torch.from_numpy(case["index"]).cuda()
    out = fx.to_torch(case["out"], dt)
    out = None if out is None else out.cuda()
    res, arg = run(src, index, case["dim"], case["reduce"], out, case["dim_size"])
    assert fx.same_bits(fx.bits_of_torch(res), case["expect"], dt), case["name"]
    if case["has_arg"]:
        assert np.array_equal(arg.cpu().numpy(), case["arg"]), case["name"]
    if out is not None:
        assert res.data_ptr() == out.data_ptr()


def _values(g, dtype, reduce, shape):
    if dtype.is_floating_point:
        if reduce == "mul":
            v = 0.9 + 0.2 * torch.rand(shape, generator=g, dtype=torch.float64)
        else:
            v = torch.randn(shape, generator=g, dtype=torch.float64) * 10
        return v.to(dtype)
    return torch.randint(-3, 4, shape, generator=g).to(dtype)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.float16, torch.bfloat16, torch.int32])
@pytest.mark.parametrize("layout", ["sorted", "unsorted", "full", "middle"])
def test_random_against_oracle(dtype, layout):
    g = torch.Generator().manual_seed(11)
    for reduce in REDUCES:
        if layout == "sorted":
            src = _values(g, dtype, reduce, (20000,))
            index = torch.sort(torch.randint(0, 700, (20000,), generator=g))[0]
            dim = 0
        elif layout == "unsorted":
            src = _values(g, dtype, reduce, (20000,))
            index = torch.randint(0, 700, (20000,), generator=g)
            dim = 0
        elif layout == "full":
            src = _values(g, dtype, reduce, (3, 3000, 5))
            index = torch.randint(0, 90, (3, 3000, 5), generator=g)
            dim = 1
        else:
            src = _values(g, dtype, reduce, (4, 3000, 7))
            index = torch.randint(0, 90, (3000,), generator=g)
            dim = 1
        res, arg = run(src.cuda(), index.cuda(), dim, reduce)
        want, warg = oracle(src, index, dim, reduce)
        check_bits(res, want, dtype)
        if warg is not None:
            assert np.array_equal(arg.cpu().numpy(), warg), (layout, reduce)


def test_sorted_and_unsorted_paths_agree_with_oracle_on_long_gaps():
    """Indices with long runs of empty outputs (filled by whole blocks) and values past the last
    element; the same data given sorted and shuffled."""
    g = torch.Generator().manual_seed(3)
    index = torch.tensor([0, 0, 5000, 5001, 5001, 90000, 90000, 90000], dtype=torch.int64)
    src = torch.randn(8, generator=g)
    for reduce in REDUCES:
        for perm in (torch.arange(8), torch.randperm(8, generator=g)):
            s, i = src[perm], index[perm]
            res, arg = run(s.cuda(), i.cuda(), 0, reduce, dim_size=200000)
            want, warg = oracle(s, i, 0, reduce, dim_size=200000)
            check_bits(res, want, torch.float32)
            if warg is not None:
                assert np.array_equal(arg.cpu().numpy(), warg)


def test_cpu_inputs_come_back_to_the_cpu_and_out_is_updated_in_place():
    src = torch.arange(10, dtype=torch.float32)
    index = torch.tensor([0, 1, 0, 1, 2, 2, 2, 3, 3, 0])
    res = tcr().scatter_sum(src, index, 0)
    assert res.device.type == "cpu"
    assert res.tolist() == [0 + 2 + 9, 1 + 3, 4 + 5 + 6, 7 + 8]
    out = torch.ones(4)
    r2 = tcr().scatter_sum(src, index, 0, out)
    assert r2 is out and out.tolist() == [12.0, 5.0, 16.0, 16.0]
    mx, arg = tcr().scatter_max(src.cuda(), index.cuda(), 0)
    assert mx.tolist() == [9.0, 3.0, 6.0, 8.0] and arg.tolist() == [9, 3, 6, 8]


def test_errors():
    src = torch.ones(5, device="cuda")
    with pytest.raises(RuntimeError):
        tcr().scatter_sum(src, torch.zeros(5, dtype=torch.int32, device="cuda"), 0)
    with pytest.raises(IndexError):
        tcr().scatter_sum(src, torch.tensor([0, 1, 2, 3, -1], device="cuda"), 0)
    with pytest.raises(IndexError):
        tcr().scatter_sum(src, torch.tensor([0, 1, 2, 3, 4], device="cuda"), 0, None, 3)
    with pytest.raises(RuntimeError):
        tcr().scatter_sum(torch.ones(2, 5, device="cuda"), torch.zeros(5, dtype=torch.int64, device="cuda"), 1,
                          torch.zeros(3, 5, device="cuda"))


def test_gradients_follow_the_reference_formulas():
    g = torch.Generator().manual_seed(5)
    src = (torch.rand(4, 300, 3, generator=g, dtype=torch.float64) + 0.5)
    index = torch.randint(0, 40, (300,), generator=g)
    index_b = index.view(1, 300, 1).expand(4, 300, 3)
    for reduce in REDUCES:
        s = src.clone().cuda().requires_grad_(True)
        res = getattr(tcr(), "scatter_" + reduce)(s, index.cuda(), 1)
        out = res[0] if isinstance(res, tuple) else res
        w = torch.randn(out.shape, generator=g, dtype=torch.float64).cuda()
        (out * w).sum().backward()
        ib = index_b.cuda()
        if reduce == "sum":
            want = torch.gather(w, 1, ib)
        elif reduce == "mean":
            count = torch.zeros(40, dtype=torch.float64).index_add_(0, index, torch.ones(300, dtype=torch.float64))
            want = torch.gather(w, 1, ib) / count.clamp(min=1).cuda()[index.cuda()].view(1, 300, 1)
        elif reduce == "mul":
            want = torch.gather(w * out.detach(), 1, ib) / s.detach()
        else:
            arg = res[1]
            want = torch.zeros(4, 301, 3, dtype=torch.float64, device="cuda").scatter_(1, arg, w)[:, :300]
        torch.testing.assert_close(s.grad, want, rtol=1e-12, atol=1e-12)


def test_neighbour_list_reduction_at_full_size():
    """Per-particle sums over the 1M-point neighbour list (rows sorted, 52M pairs): counts equal
    the CSR row lengths exactly, and sampled rows equal a serial float32 fold."""
    import bench
    tc = tcr()
    pos, sup = bench.make_workload()
    p, h = pos.cuda(), sup.cuda()
    dom = tc.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.zeros(3, dtype=torch.bool), 3)
    adj = tc.radiusSearch(tc.PointCloud(p, h), None, mode="symmetric", domain=dom, algorithm="compact", format="coo")
    csr = tc.radiusSearch(tc.PointCloud(p, h), None, mode="symmetric", domain=dom, algorithm="compact", format="csr")
    n = p.shape[0]
    ones = torch.ones(adj.row.numel(), device="cuda")
    counts = tc.scatter_sum(ones, adj.row, 0, None, n)
    assert torch.equal(counts, csr.rowEntries.float())
    vals = torch.rand(adj.row.numel(), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    sums = tc.scatter_sum(vals, adj.row, 0, None, n)
    rows = torch.randint(0, n, (64,), generator=torch.Generator().manual_seed(2))
    indptr = csr.indptr.cpu().numpy()
    v = vals.cpu().numpy()
    row_of = adj.row.cpu().numpy()
    starts = np.searchsorted(row_of, rows.numpy(), side="left")
    ends = np.searchsorted(row_of, rows.numpy(), side="right")
    for r, a, b in zip(rows.tolist(), starts, ends):
        assert b - a == indptr[r + 1] - indptr[r]
        acc = np.cumsum(v[a:b], dtype=np.float32)[-1] if b > a else np.float32(0)
        assert np.float32(sums[r].item()) == acc


def test_known_size_paths_fall_back_for_unsorted_and_reject_out_of_range():
    """With the output size known the index is first taken in its own order; an index that
    descends (here one alternating between the ends, whose runs would overlap) falls back to the
    sorted path, and an index outside [0, N) leaves a given out untouched."""
    g = torch.Generator().manual_seed(8)
    N = 100000
    index = torch.zeros(20000, dtype=torch.int64)
    index[1::2] = N - 1
    src = torch.randn(20000, generator=g)
    for reduce in REDUCES:
        res, arg = run(src.cuda(), index.cuda(), 0, reduce, dim_size=N)
        want, warg = oracle(src, index, 0, reduce, dim_size=N)
        check_bits(res, want, torch.float32)
        if warg is not None:
            assert np.array_equal(arg.cpu().numpy(), warg)
    out = torch.full((10,), 7.0, device="cuda")
    bad = torch.tensor([0, 3, 10], device="cuda")
    with pytest.raises(IndexError):
        tcr().scatter_sum(torch.ones(3, device="cuda"), bad, 0, out)
    assert torch.equal(out, torch.full((10,), 7.0, device="cuda"))


@pytest.mark.parametrize("shape,dim", [((3, 5000), 1), ((5000, 6), 0), ((2, 5000, 40), 1)])
def test_sorted_index_with_known_size_and_batches_or_features(shape, dim):
    g = torch.Generator().manual_seed(12)
    E = shape[dim]
    index = torch.sort(torch.randint(0, 300, (E,), generator=g))[0]
    for dtype in (torch.float32, torch.bfloat16, torch.int64):
        for reduce in REDUCES:
            src = _values(g, dtype, reduce, shape)
            res, arg = run(src.cuda(), index.cuda(), dim, reduce, dim_size=310)
            want, warg = oracle(src, index, dim, reduce, dim_size=310)
            check_bits(res, want, dtype)
            if warg is not None:
                assert np.array_equal(arg.cpu().numpy(), warg)
