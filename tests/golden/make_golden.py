"""Generates the golden fixtures from the reference package itself.

Run where the reference checkout exists (named by --reference or TCR_REFERENCE) and its CPU
operators have been built by ``oracle/build_ref.py``:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py --reference <checkout>

For every case it calls the reference's public ``torchCompactRadius.radiusSearch(...,
algorithm='compact')`` with an explicit ``DomainDescription`` and records, per case, the SHA-256
of the generated inputs, the pair count, the per-row counts and the SHA-256 of the
canonically sorted (row, col) pairs; for the small scripts/test.py grid it also stores the
full CSR so a failing test can show the difference.  Output: ``reference_cases.json`` and
``reference_cases.npz`` next to this file.
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import cases  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TCR_REFERENCE"),
                    help="reference checkout (default: the TCR_REFERENCE environment variable)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set TCR_REFERENCE")
    sys.path[:0] = [os.path.join(REPO, "oracle", "_ref"), os.path.join(a.reference, "src")]
    import torch
    import torchCompactRadius as tcr
    from torchCompactRadius.util import DomainDescription, PointCloud

    def run(xq, hq, xr, hr, dmin, dmax, per, mode, L, fmt="csr"):
        dom = DomainDescription(torch.tensor(dmin), torch.tensor(dmax), torch.tensor(per, dtype=torch.bool), len(dmin))
        q = PointCloud(torch.tensor(xq), None if hq is None else torch.tensor(hq))
        r = None if xr is None else PointCloud(torch.tensor(xr), None if hr is None else torch.tensor(hr))
        out = tcr.radiusSearch(q, r, mode=mode, domain=dom, hashMapLength=L, algorithm="compact", format=fmt)
        indptr = out.indptr.numpy().astype(np.int64)
        rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
        return rows, out.indices.numpy(), out.indptr.numpy(), out.rowEntries.numpy()

    meta = {"reference": "torchCompactRadius " + tcr.__version__, "cases": []}
    arrays = {}

    # scripts/test.py:84-118 fixture and its known answers
    for reduced in (False, True):
        q, ref, h = cases.testpy_grid(reduced)
        for per in (True, False):
            for mode in cases.MODES:
                name = f"testpy_{'reduced' if reduced else 'full'}_{'periodic' if per else 'open'}_{mode}"
                hq = np.full(len(q), h, np.float32)
                hr = np.full(len(ref), h, np.float32)
                rows, cols, indptr, entries = run(q, hq, ref, hr, [-1.0, -1.0], [1.0, 1.0], [per, per], mode, 4096)
                meta["cases"].append(dict(kind="testpy", name=name, reduced=reduced, periodic=per, mode=mode, L=4096,
                                          input_sha=cases.sha(q, ref, np.float32(h)), npairs=int(len(cols)),
                                          pair_sha=cases.pair_sha(rows, cols), indptr_sha=cases.sha(indptr),
                                          row_min=int(entries.min()), row_max=int(entries.max())))
                if mode == "gather":
                    arrays[name + "/indptr"] = indptr.astype(np.int32)
                    r_, c_ = cases.canonical(rows, cols)
                    arrays[name + "/cols"] = c_.astype(np.int16)
    # the plain 2D periodic workload
    pos, sup = cases.cfg1_inputs()
    rows, cols, indptr, entries = run(pos, sup, None, None, [-1.0, -1.0], [1.0, 1.0], [True, True], "gather", 4096)
    meta["cases"].append(dict(kind="cfg1", name="cfg1_2d_periodic_gather", mode="gather", L=4096,
                              input_sha=cases.sha(pos, sup), npairs=int(len(cols)),
                              pair_sha=cases.pair_sha(rows, cols), indptr_sha=cases.sha(indptr)))
    arrays["cfg1_2d_periodic_gather/counts"] = entries.astype(np.int16)
    # seeded random clouds
    for name, kw, mode, L in cases.random_cases():
        x, hx, y, hy, dmin, dmax, per = cases.random_case(**kw)
        rows, cols, indptr, entries = run(x, hx, y, hy, dmin.tolist(), dmax.tolist(), per.tolist(), mode, L)
        meta["cases"].append(dict(kind="random", name=name, params=kw, mode=mode, L=L,
                                  input_sha=cases.sha(x, hx, y, hy), npairs=int(len(cols)),
                                  pair_sha=cases.pair_sha(rows, cols), indptr_sha=cases.sha(indptr)))
        arrays[name + "/counts"] = entries.astype(np.int16)
        print(f"{name:40s} P={len(cols)}")
    with open(os.path.join(HERE, "reference_cases.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "reference_cases.npz"), **arrays)
    print(len(meta["cases"]), "cases written")


if __name__ == "__main__":
    main()
