"""The float64 brute-force oracle against the reference's own double search (CPU only)."""
import numpy as np
import pytest

import cases
import f64_fixtures as fx
from oracle import search64

CASES = fx.load()


@pytest.mark.parametrize("case", CASES, ids=[fx.name(c) for c in CASES])
def test_oracle_matches_reference_double_search(case):
    x, hx, y, hy, lo, hi, per = fx.inputs(case)
    row, col = search64.radius_search(x, hx, y, hy, lo, hi, per, case["mode"])
    assert row.size == case["pairs"]
    assert cases.pair_sha(row, col) == case["pair_sha"]
    n = x.shape[0]
    assert np.array_equal(np.bincount(row, minlength=n).astype(np.int32), case["row_counts"])


def test_double_and_float_searches_differ_on_the_lattice():
    """On the lattice cases many pairs sit at the threshold: the double result is not the float
    one, so these fixtures pin the double arithmetic itself."""
    import torch
    c = next(c for c in CASES if c["lattice"] and c["dim"] == 2)
    x, hx, y, hy, lo, hi, per = fx.inputs(c)
    row, col = search64.radius_search(x.astype(np.float32).astype(np.float64),
                                      hx.astype(np.float32).astype(np.float64), None, None, lo, hi, per, c["mode"])
    assert cases.pair_sha(row, col) != c["pair_sha"] or row.size != c["pairs"]
