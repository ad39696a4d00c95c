"""The scatter oracle against the reference's own outputs (CPU only)."""
import numpy as np
import pytest

import scatter_fixtures as fx
from oracle import scatter as oracle_scatter
from torchcompactradius_b200.scatter import broadcast

CASES = fx.load()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_bits(case):
    import torch
    dt = case["dtype"]
    src = fx.to_numpy(case["src"], dt)
    index = case["index"]
    dim = case["dim"]
    # the reference's own broadcast of the index, on the CPU
    index_b = broadcast(torch.from_numpy(index), torch.empty(src.shape), dim + src.ndim if dim < 0 else dim).numpy()
    out = fx.to_numpy(case["out"], dt)
    res, arg = oracle_scatter.scatter(src, index_b, dim, case["reduce"], out=out, dim_size=case["dim_size"],
                                      bf16=(dt == "bfloat16"))
    assert fx.same_bits(fx.bits_of_numpy(res, dt), case["expect"], dt), case["name"]
    if case["has_arg"]:
        assert np.array_equal(arg, case["arg"]), case["name"]


def test_fixture_coverage():
    """Every reduce meets every element type, and the special layouts are present."""
    seen = {(c["dtype"], c["reduce"]) for c in CASES}
    for dt in ("float32", "float64", "float16", "bfloat16", "int64", "int32", "int16", "int8", "uint8"):
        for r in ("sum", "mean", "mul", "min", "max"):
            assert (dt, r) in seen
    names = " ".join(c["name"] for c in CASES)
    for kind in ("sorted_", "full_", "lastdim_", "out_", "dimsize_", "empty_", "specials_", "long_", "wrap_"):
        assert kind in names


def test_oracle_order_matters_for_half_sums():
    """A fold in a different order changes float16 sums: the fixtures pin the order, not just the
    values (a reassociating device reduction would fail them)."""
    case = next(c for c in CASES if c["name"] == "long_float16_sum")
    src = fx.to_numpy(case["src"], "float16")
    idx = case["index"]
    res, _ = oracle_scatter.scatter(src[::-1].copy(), idx[::-1].copy(), 0, "sum")
    assert not fx.same_bits(fx.bits_of_numpy(res, "float16"), case["expect"], "float16")
