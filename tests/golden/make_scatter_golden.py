"""Generates the scatter fixtures from the reference's own compiled operators.

Run where the reference's CPU operators have been built by ``oracle/build_ref.py``:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_scatter_golden.py

Every case calls ``torch.ops.torchCompactRadius_cpu.scatter_<reduce>(src, index, dim, out,
dim_size)`` (src/torchCompactRadius/cppSrc/sparseOperations/scatterWrapper.cpp:225-266) on seeded
inputs and stores the inputs and the reference's outputs as raw bits (bfloat16 as uint16) in
``scatter_cases.npz`` next to this file; ``meta`` holds one JSON record per case.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

DTYPES = ["float32", "float64", "float16", "bfloat16", "int64", "int32", "int16", "int8", "uint8"]
REDUCES = ["sum", "mean", "mul", "min", "max"]


def raw(t):
    """A tensor's values as a numpy array of the same bits (bfloat16 -> uint16)."""
    import torch
    if t.dtype == torch.bfloat16:
        return t.contiguous().view(torch.int16).numpy().view(np.uint16).copy()
    return t.contiguous().numpy().copy()


def values(g, dtype, reduce, shape):
    """Seeded values for one case: products stay near 1, integers small (so wrap-around is rare
    but reachable), floating sums get magnitudes that make the order of addition matter."""
    import torch
    t = getattr(torch, dtype)
    if dtype.startswith("float") or dtype == "bfloat16":
        if reduce == "mul":
            v = 0.5 + torch.rand(shape, generator=g, dtype=torch.float64)
        else:
            v = torch.randn(shape, generator=g, dtype=torch.float64) * 3.0 * torch.exp(
                torch.randn(shape, generator=g, dtype=torch.float64))
        return v.to(t)
    lo, hi = (0, 6) if dtype == "uint8" else (-5, 6)
    if reduce == "mul":
        lo, hi = (0, 3) if dtype == "uint8" else (-2, 3)
    return torch.randint(lo, hi, shape, generator=g, dtype=torch.int64).to(t)


def main():
    import torch
    from oracle import ref_pipeline
    ops = ref_pipeline.ops()
    g = torch.Generator().manual_seed(7)
    cases = []

    def add(name, src, index, dim, reduce, out=None, dim_size=None):
        fn = getattr(ops, "scatter_" + reduce)
        o = None if out is None else out.clone()
        res = fn(src, index, dim, o, dim_size)
        arg = None
        if reduce in ("min", "max"):
            res, arg = res
        cases.append(dict(name=name, dtype=str(src.dtype).replace("torch.", ""), reduce=reduce, dim=dim,
                          dim_size=dim_size, src=raw(src), index=index.numpy().copy(),
                          out=None if out is None else raw(out), expect=raw(res),
                          arg=None if arg is None else arg.numpy().copy()))

    for dt in DTYPES:  # 1-D, unsorted index
        for r in REDUCES:
            src = values(g, dt, r, (300,))
            idx = torch.randint(0, 40, (300,), generator=g)
            add(f"1d_{dt}_{r}", src, idx, 0, r)
    for dt in ("float32", "float16", "bfloat16", "int32"):  # index along the middle dimension
        for r in REDUCES:
            src = values(g, dt, r, (3, 200, 4))
            idx = torch.randint(0, 25, (200,), generator=g)
            add(f"mid_{dt}_{r}", src, idx, 1, r)
    for dt in ("float32", "float64", "bfloat16"):  # non-decreasing index (a neighbour list's rows)
        for r in REDUCES:
            src = values(g, dt, r, (500,))
            idx = torch.sort(torch.randint(0, 60, (500,), generator=g))[0]
            add(f"sorted_{dt}_{r}", src, idx, 0, r)
    for dt in ("float32", "int64"):  # an index of src's full shape
        for r in REDUCES:
            src = values(g, dt, r, (4, 50, 3))
            idx = torch.randint(0, 10, (4, 50, 3), generator=g)
            add(f"full_{dt}_{r}", src, idx, 1, r)
    for r in REDUCES:  # the last dimension, named as -1
        src = values(g, "float32", r, (5, 60))
        idx = torch.randint(0, 12, (60,), generator=g)
        add(f"lastdim_float32_{r}", src, idx, -1, r)
    for dt in ("float32", "int32"):  # reduced into a given out
        for r in REDUCES:
            src = values(g, dt, r, (100,))
            idx = torch.randint(0, 15, (100,), generator=g)
            out = values(g, dt, r, (15,))
            add(f"out_{dt}_{r}", src, idx, 0, r, out=out)
    for dt in ("float32", "float16"):  # dim_size past the largest index: empty outputs
        for r in REDUCES:
            src = values(g, dt, r, (80,))
            idx = torch.randint(0, 10, (80,), generator=g)
            add(f"dimsize_{dt}_{r}", src, idx, 0, r, dim_size=16)
    for r in REDUCES:  # no elements at all
        add(f"empty_float32_{r}", torch.zeros(0), torch.zeros(0, dtype=torch.int64), 0, r, dim_size=5)
    specials = torch.tensor([1.0, 1.0, -2.0, float("nan"), float("inf"), -float("inf"), 3.4028234663852886e38,
                             -3.4028234663852886e38, 0.0, -0.0, 2.0, 2.0, float("nan"), 5.0, 5.0, -7.0])
    sidx = torch.tensor([0, 0, 0, 1, 1, 2, 3, 4, 5, 5, 6, 6, 6, 7, 7, 7])
    for r in REDUCES:  # ties, NaN, infinities, the float extremes
        add(f"specials_float32_{r}", specials, sidx, 0, r)
    for dt in ("float16", "bfloat16"):  # long folds: rounding order and saturating counts
        for r in ("sum", "mean"):
            src = (torch.rand((3000,), generator=g, dtype=torch.float64) * 40.0).to(getattr(torch, dt))
            idx = torch.randint(0, 2, (3000,), generator=g)
            add(f"long_{dt}_{r}", src, idx, 0, r)
    for r in ("sum", "mean", "mul"):  # 8-bit wrap-around, counts past 127
        src = torch.randint(-3, 4, (300,), generator=g, dtype=torch.int64).to(torch.int8)
        idx = torch.zeros(300, dtype=torch.int64)
        add(f"wrap_int8_{r}", src, idx, 0, r)

    arrays = {}
    meta = []
    for i, c in enumerate(cases):
        rec = {k: c[k] for k in ("name", "dtype", "reduce", "dim", "dim_size")}
        rec["has_out"] = c["out"] is not None
        rec["has_arg"] = c["arg"] is not None
        meta.append(rec)
        for k in ("src", "index", "out", "expect", "arg"):
            if c[k] is not None:
                arrays[f"c{i}_{k}"] = c[k]
    arrays["meta"] = np.array(json.dumps(meta))
    path = os.path.join(HERE, "scatter_cases.npz")
    np.savez_compressed(path, **arrays)
    print(f"{len(cases)} cases -> {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
