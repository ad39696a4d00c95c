"""The C oracle pinned against the reference's own outputs (golden fixtures) and known answers.

The fixtures were produced by the reference package itself (tests/golden/make_golden.py);
scripts/test.py:84-118 of the reference gives the known answers of the 32x32 grid.
"""
import numpy as np
import pytest

import cases
from oracle import compact


def _inputs(c):
    if c["kind"] == "testpy":
        q, ref, h = cases.testpy_grid(c["reduced"])
        assert cases.sha(q, ref, np.float32(h)) == c["input_sha"]
        per = [c["periodic"]] * 2
        return (q, np.full(len(q), h, np.float32), ref, np.full(len(ref), h, np.float32),
                np.array([-1, -1], np.float32), np.array([1, 1], np.float32), per)
    if c["kind"] == "cfg1":
        pos, sup = cases.cfg1_inputs()
        assert cases.sha(pos, sup) == c["input_sha"]
        return pos, sup, None, None, np.array([-1, -1], np.float32), np.array([1, 1], np.float32), [True, True]
    x, hx, y, hy, dmin, dmax, per = cases.random_case(**c["params"])
    assert cases.sha(x, hx, y, hy) == c["input_sha"]
    return x, hx, y, hy, dmin, dmax, per


def test_known_answers_scripts_test_py(golden):
    meta, arrays = golden
    by = {c["name"]: c for c in meta["cases"]}
    for mode in cases.MODES:
        c = by[f"testpy_full_periodic_{mode}"]
        assert c["npairs"] == 46080 and c["row_min"] == c["row_max"] == 45
        c = by[f"testpy_full_open_{mode}"]
        assert c["npairs"] == 41580 and (c["row_min"], c["row_max"]) == (15, 45)
        for per in ("periodic", "open"):
            c = by[f"testpy_reduced_{per}_{mode}"]
            assert c["npairs"] == 11520 and c["row_min"] == c["row_max"] == 45


@pytest.mark.parametrize("idx", range(61))
def test_oracle_matches_reference_fixture(golden, idx):
    meta, arrays = golden
    c = meta["cases"][idx]
    xq, hq, xr, hr, dmin, dmax, per = _inputs(c)
    r = compact.radius_search(xq, hq, xr, hr, dmin, dmax, per, c["mode"], c["L"])
    assert len(r.col) == c["npairs"]
    assert cases.pair_sha(r.row, r.col) == c["pair_sha"]
    indptr = r.offsets.astype(np.int32)
    assert cases.sha(indptr) == c["indptr_sha"]
    key = c["name"] + "/cols"
    if key in arrays:
        _, cc = cases.canonical(r.row, r.col)
        np.testing.assert_array_equal(cc, arrays[key].astype(np.int64))


def test_hash_matches_reference_formula():
    # hashing.h:20-34: uint32 wrap-around, negative coordinates reinterpret as unsigned
    for cell, L in [((3, -2, 7), 4096), ((-1, 5), 7), ((12,), 10), ((-3,), 10), ((2**20, 2**21, -2**22), 65537)]:
        p = [73856093, 19349663, 83492791]
        if len(cell) == 1:
            exp = (cell[0] & 0xFFFFFFFF) % L
        else:
            exp = (sum((c & 0xFFFFFFFF) * p[d] for d, c in enumerate(cell)) & 0xFFFFFFFF) % L
        assert compact.hash_cell(cell, L) == exp


def test_wrap_matches_torch_remainder():
    import torch
    rng = np.random.default_rng(5)
    x = (rng.random(20000) * 8 - 4).astype(np.float32)
    x[:4] = [-1.0, 1.0, np.float32(1) - np.float32(2 ** -24), np.float32(-1) - np.float32(2 ** -23)]
    lo, hi = np.float32(-1.0), np.float32(1.0)
    t = torch.remainder(torch.tensor(x) - torch.tensor(lo), torch.tensor(hi) - torch.tensor(lo)) + torch.tensor(lo)
    got = np.array([compact.wrap(v, lo, hi) for v in x], np.float32)
    np.testing.assert_array_equal(got, t.numpy())


def test_compute_hcell_matches_torch_expression():
    import torch
    rng = np.random.default_rng(7)
    for _ in range(300):
        dim = int(rng.integers(1, 4))
        lo = (rng.random(dim) * -2).astype(np.float32)
        hi = (lo + 0.5 + rng.random(dim) * 3).astype(np.float32)
        hmax = np.float32(rng.random() * 0.3 + 1e-3)
        # util.py:28-79, evaluated with torch float32 tensors
        qMin, qMax, ref = torch.tensor(lo), torch.tensor(hi), torch.tensor(hmax)
        ext = qMax - qMin
        nc = torch.floor(ext / ref)
        h = ext / nc
        if torch.any(ext / h - nc > 0):
            nc -= 1
            h = ext / nc
        if torch.any(torch.ceil(ext / h) > ext / h):
            h = h * (1e-4 + 1)
        exp = torch.max(h)
        got, cnt = compact.compute_hcell(lo, hi, hmax)
        assert np.float32(got) == exp.numpy(), (lo, hi, hmax)
        np.testing.assert_array_equal(cnt, torch.ceil(ext / exp).to(torch.int32).numpy())


def test_brute_force_agrees_with_compact_on_open_domain():
    x, hx, y, hy, dmin, dmax, per = cases.random_case(seed=3, dim=3, n=1500, nref=None, hscale=0.15,
                                                      extent=[2, 2, 2], periodic=[False] * 3)
    for mode in cases.MODES:
        a = compact.radius_search(x, hx, None, None, dmin, dmax, per, mode, 4096)
        b = compact.brute_force(x, hx, None, None, dmin, dmax, per, mode)
        assert cases.pair_sha(a.row, a.col) == cases.pair_sha(b.row, b.col)
