"""Host-side pieces of the float64 search (CPU only): the double wrap and cell size against the
reference's own torch operations restated in the oracle, and the cell size's coverage guarantee."""
import math

import numpy as np
import pytest
import torch

from oracle import ref_pipeline, search64 as oracle64
from torchcompactradius_b200.search64 import compute_h64, wrap64


@pytest.mark.parametrize("hmax", [0.0448, 0.1, 0.25, 0.4, 2.0 / 7, 0.333333, 1.5, 2.5])
@pytest.mark.parametrize("lo,hi", [([-1.0] * 3, [1.0] * 3), ([0.0, -2.0, 0.5], [1.0, 3.0, 0.75])])
def test_compute_h64_equals_the_reference_restatement_in_double(hmax, lo, hi):
    want = ref_pipeline.compute_h(torch.tensor(lo, dtype=torch.float64), torch.tensor(hi, dtype=torch.float64),
                                  torch.tensor(hmax, dtype=torch.float64))
    got = compute_h64(lo, hi, hmax)
    w = float(want)
    assert (math.isnan(got) and math.isnan(w)) or got == w
    if math.isfinite(got) and got > 0:
        assert got >= hmax  # every support fits in one cell


def test_wrap64_equals_the_oracle_wrap():
    rng = np.random.default_rng(3)
    x = rng.uniform(-3.0, 3.0, (5000, 3))
    lo, hi, per = [-1.0, -0.5, 0.0], [1.0, 0.75, 2.0], [True, False, True]
    mask = 0b101
    got = wrap64(torch.tensor(x), lo, hi, mask).numpy()
    want = oracle64.wrap(x, lo, hi, per)
    assert np.array_equal(got, want)
    assert np.all((got[:, 0] >= -1.0) & (got[:, 0] < 1.0)) and np.array_equal(got[:, 1], x[:, 1])
