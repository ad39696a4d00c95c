"""Input generators for the golden fixtures (shared by make_golden.py and the tests).

Every case is regenerated from a seed with numpy's PCG64 (stable across platforms); the
fixture stores the SHA-256 of the generated input bytes so a drifting generator is caught
before any output is compared.
"""
import hashlib

import numpy as np

MODES = ["gather", "scatter", "symmetric", "superSymmetric"]


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        if a is None:
            h.update(b"none")
        else:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def canonical(row, col):
    """Pairs sorted by (row, col) as int64."""
    row = np.asarray(row, np.int64)
    col = np.asarray(col, np.int64)
    o = np.lexsort((col, row))
    return row[o], col[o]


def pair_sha(row, col):
    r, c = canonical(row, col)
    return sha(r, c)


def volume_to_support(volume, k, dim):
    """util.py:5-26 volumeToSupport in float64."""
    if dim == 1:
        return k * volume / 2
    if dim == 2:
        return float(np.sqrt(k * volume / np.pi))
    return float(np.power(k * volume / np.pi * 3 / 4, 1 / 3))


def testpy_grid(reduced):
    """scripts/test.py:31-68 generateNeighborTestData(nx=32, 50 neighbours, dim=2, [-1,1]^2).

    Returns (query, reference, h).  The reduced query set is the central 16x16 grid."""
    import torch
    dim, nx, k = 2, 32, 50
    dmin = torch.tensor([-1.0] * dim)
    dmax = torch.tensor([1.0] * dim)
    extent = dmax - dmin
    dx = float(torch.min(extent).item()) / nx
    ny = int(1 // dx)
    h = volume_to_support(dx ** dim, k, dim)
    axes = [torch.linspace(float(dmin[d]) + dx / 2, float(dmax[d]) - dx / 2, int((extent[d] - dx) / dx) + 1)
            for d in range(dim)]
    g = torch.meshgrid(*axes, indexing="xy")
    pos = torch.stack(g, dim=-1).reshape(-1, dim).numpy().astype(np.float32)
    yax = [torch.linspace(-0.5 + dx / 2, 0.5 - dx / 2, ny) for _ in range(dim)]
    g = torch.meshgrid(*yax, indexing="xy")
    y = torch.stack(g, dim=-1).reshape(-1, dim).numpy().astype(np.float32)
    q = y if reduced else pos
    return q, pos, np.float32(h)


def cfg1_inputs():
    """2D periodic 64x64 jittered grid on [-1,1]^2 (the plain CPU-runnable workload).

    Cell-centred grid, dx = 2/64, jitter U(-0.1dx, 0.1dx) per coordinate from numpy PCG64
    seed 0, uniform support h = sqrt(32 dx^2 / pi)."""
    n = 64
    dx = 2.0 / n
    g = (np.arange(n) + 0.5) * dx - 1.0
    X, Y = np.meshgrid(g, g, indexing="xy")
    pos = np.stack([X.ravel(), Y.ravel()], 1).astype(np.float32)
    rng = np.random.default_rng(0)
    pos = (pos + ((rng.random(pos.shape) * 2 - 1) * 0.1 * dx).astype(np.float32)).astype(np.float32)
    h = np.float32(np.sqrt(32 * dx * dx / np.pi))
    sup = np.full(n * n, h, np.float32)
    return pos, sup


def random_case(seed, dim, n, nref, hscale, extent, periodic):
    """Uniform random cloud(s) in [0, extent] per dim with supports hscale*U(0.5, 1.5).

    nref=None means the query cloud doubles as the reference cloud.  A few points are placed
    within one ulp-scale distance of the upper domain bound to exercise the periodic wrap."""
    rng = np.random.default_rng(seed)
    ext = np.asarray(extent, np.float32)
    x = (rng.random((n, dim)) * ext).astype(np.float32)
    hx = (hscale * (0.5 + rng.random(n))).astype(np.float32)
    k = min(8, n)
    x[:k] = (ext - (rng.random((k, dim)) * 1e-6).astype(np.float32)).astype(np.float32)
    if nref is None:
        y, hy = None, None
    else:
        y = (rng.random((nref, dim)) * ext).astype(np.float32)
        hy = (hscale * (0.5 + rng.random(nref))).astype(np.float32)
    return x, hx, y, hy, np.zeros(dim, np.float32), ext.astype(np.float32), np.asarray(periodic, bool)


def random_cases():
    """(name, kwargs for random_case, mode, hashMapLength) for the golden set."""
    out = []
    for dim in (1, 2, 3):
        n = {1: 1500, 2: 3000, 3: 6000}[dim]
        hs = {1: 0.004, 2: 0.06, 3: 0.12}[dim]
        for pi, per in enumerate(([False] * dim, [True] * dim, [True] + [False] * (dim - 1))):
            for mi, mode in enumerate(MODES):
                seed = 1000 + 100 * dim + 10 * pi + mi
                out.append((f"d{dim}_p{''.join('1' if p else '0' for p in per)}_{mode}",
                            dict(seed=seed, dim=dim, n=n, nref=None, hscale=hs, extent=[2.0] * dim, periodic=per),
                            mode, 4096))
    # distinct query / reference clouds in a non-cubic periodic box, and a tiny hash table
    for mi, mode in enumerate(MODES):
        for L in (4096, 7):
            out.append((f"noncubic_qr_{mode}_L{L}",
                        dict(seed=2000 + mi, dim=3, n=2500, nref=3500, hscale=0.1, extent=[2.0, 1.5, 1.0],
                             periodic=[True, True, True]), mode, L))
    return out
