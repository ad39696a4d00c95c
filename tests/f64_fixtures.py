"""Loads tests/golden/f64_cases.npz (made by tests/golden/make_f64_golden.py from the reference's
own double search) and regenerates each case's inputs."""
import json
import os

import numpy as np

import cases
import f64_cases

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "f64_cases.npz")


def load():
    z = np.load(PATH)
    meta = json.loads(str(z["meta"]))
    out = []
    for k, m in enumerate(meta):
        c = dict(m)
        c["row_counts"] = z[f"c{k}_row_counts"]
        out.append(c)
    return out


def inputs(c):
    x, hx, y, hy, lo, hi, per = f64_cases.inputs_of(c)
    assert cases.sha(x, hx, y, hy) == c["input_sha"], "the input generator drifted"
    return x, hx, y, hy, lo, hi, per


def name(c):
    return f"d{c['dim']}_{c['mode']}_{''.join('p' if p else 'o' for p in c['periodic'])}" + \
           ("_lattice" if c["lattice"] else "") + ("_xy" if c["nref"] else "")
