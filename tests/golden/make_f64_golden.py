"""Generates the float64 fixtures from the reference package itself (double inputs).

Run where the reference checkout exists and its CPU operators are built by ``oracle/build_ref.py``:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_f64_golden.py --reference <checkout>

For every case of ``f64_cases.f64_cases()`` it calls the reference's public
``torchCompactRadius.radiusSearch(..., algorithm='compact', format='csr')`` with float64 positions,
supports and domain, and stores the SHA-256 of the inputs, the pair count, the per-row counts and
the SHA-256 of the canonically sorted pairs in ``f64_cases.npz`` next to this file.
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
import f64_cases  # noqa: E402


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

    meta, arrays = [], {}
    for k, c in enumerate(f64_cases.f64_cases()):
        x, hx, y, hy, lo, hi, per = f64_cases.inputs_of(c)
        dom = DomainDescription(torch.tensor(lo, dtype=torch.float64), torch.tensor(hi, dtype=torch.float64),
                                torch.tensor(per, dtype=torch.bool), len(lo))
        q = PointCloud(torch.tensor(x), torch.tensor(hx))
        r = None if y is None else PointCloud(torch.tensor(y), torch.tensor(hy))
        adj = tcr.radiusSearch(q, r, mode=c["mode"], domain=dom, algorithm="compact", format="csr")
        indptr = adj.indptr.numpy().astype(np.int64)
        rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
        rec = dict(c)
        rec.update(input_sha=cases.sha(x, hx, y, hy), pairs=int(adj.indices.numel()),
                   pair_sha=cases.pair_sha(rows, adj.indices.numpy()))
        meta.append(rec)
        arrays[f"c{k}_row_counts"] = adj.rowEntries.numpy().astype(np.int32)
        print(f"case {k}: dim {c['dim']} {c['mode']} periodic {c['periodic']} lattice {c['lattice']}: "
              f"{rec['pairs']} pairs")
    arrays["meta"] = np.array(json.dumps(meta))
    path = os.path.join(HERE, "f64_cases.npz")
    np.savez_compressed(path, **arrays)
    print(f"{len(meta)} cases -> {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
