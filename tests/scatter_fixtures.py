"""Loads tests/golden/scatter_cases.npz (made by tests/golden/make_scatter_golden.py from the
reference's compiled scatter operators) and compares results bit for bit."""
import json
import os

import numpy as np
import torch

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scatter_cases.npz")


def load():
    z = np.load(PATH)
    meta = json.loads(str(z["meta"]))
    cases = []
    for i, m in enumerate(meta):
        c = dict(m)
        for k in ("src", "index", "out", "expect", "arg"):
            key = f"c{i}_{k}"
            c[k] = z[key] if key in z.files else None
        cases.append(c)
    return cases


def to_torch(a, dtype):
    """Fixture bits -> tensor of the case's dtype."""
    if a is None:
        return None
    if dtype == "bfloat16":
        return torch.from_numpy(a.view(np.int16).copy()).view(torch.bfloat16)
    return torch.from_numpy(np.array(a, copy=True))


def to_numpy(a, dtype):
    """Fixture bits -> numpy values for the oracle (bfloat16 widened to float32)."""
    if a is None:
        return None
    if dtype == "bfloat16":
        return (a.astype(np.uint32) << 16).view(np.float32)
    return np.array(a, copy=True)


def bits_of_numpy(a, dtype):
    """Oracle values -> the fixture's bit representation."""
    if dtype == "bfloat16":
        return (np.asarray(a, np.float32).view(np.uint32) >> 16).astype(np.uint16)
    return np.asarray(a)


def bits_of_torch(t):
    t = t.detach().cpu().contiguous()
    if t.dtype == torch.bfloat16:
        return t.view(torch.int16).numpy().view(np.uint16)
    return t.numpy()


def same_bits(got, want, dtype):
    """Equal bit for bit, except that any NaN equals any NaN (payloads differ between libraries)."""
    got, want = np.asarray(got), np.asarray(want)
    if got.shape != want.shape:
        return False
    if dtype == "bfloat16":
        g = (got.astype(np.uint32) << 16).view(np.float32)
        w = (want.astype(np.uint32) << 16).view(np.float32)
        both_nan = np.isnan(g) & np.isnan(w)
        return bool(np.all((got == want) | both_nan))
    if got.dtype.kind == "f":
        both_nan = np.isnan(got) & np.isnan(want)
        return bool(np.all((got.view(np.uint8 if got.itemsize == 1 else f"u{got.itemsize}") ==
                            want.view(np.uint8 if want.itemsize == 1 else f"u{want.itemsize}")) | both_nan))
    return bool(np.array_equal(got, want))
