"""Float64 input generators for the double-search fixtures (shared by make_f64_golden.py and the
tests).  Every case is regenerated from a seed with numpy's PCG64; the fixture stores the SHA-256
of the generated inputs."""
import numpy as np

from cases import sha

MODES = ["gather", "scatter", "symmetric", "superSymmetric"]


def f64_case(seed, dim, n, nref, k, periodic, lattice=False):
    """n query / nref reference points (nref 0: the query cloud itself) in [-1, 1]^dim, supports
    for about k neighbours varying by +-10%.  With
    lattice, points sit on a grid of spacing exactly a tenth of the support, so many pairs lie at
    distances within rounding of the threshold."""
    rng = np.random.default_rng(seed)
    lo = -np.ones(dim)
    hi = np.ones(dim)
    vol = 2.0 ** dim / n
    h0 = {1: k * vol / 2, 2: np.sqrt(k * vol / np.pi), 3: np.cbrt(3 * k * vol / (4 * np.pi))}[dim]
    if lattice:
        m = int(round(n ** (1 / dim)))
        axes = [np.arange(m) * (h0 / 10.0) - 1.0 for _ in range(dim)]
        g = np.meshgrid(*axes, indexing="ij")
        x = np.stack([a.reshape(-1) for a in g], 1).astype(np.float64)
        hx = np.full(x.shape[0], h0, np.float64)
    else:
        x = rng.uniform(-1.0, 1.0, (n, dim))
        hx = h0 * rng.uniform(0.9, 1.1, n)
    if nref:
        y = rng.uniform(-1.0, 1.0, (nref, dim))
        hy = h0 * rng.uniform(0.9, 1.1, nref)
    else:
        y, hy = None, None
    return x, hx, y, hy, lo, hi, np.asarray(periodic, bool)


def f64_cases():
    """(params) of every fixture case."""
    out = []
    seed = 100
    for dim in (1, 2, 3):
        for periodic in ([False] * dim, [True] * dim, [True] + [False] * (dim - 1)):
            for mode in MODES:
                seed += 1
                out.append(dict(seed=seed, dim=dim, n=1500 if dim > 1 else 800, nref=0, k=30 if dim > 1 else 12,
                                periodic=periodic, mode=mode, lattice=False))
    for mode in MODES:
        seed += 1
        out.append(dict(seed=seed, dim=3, n=1200, nref=900, k=40, periodic=[True, False, True], mode=mode,
                        lattice=False))
    for dim in (2, 3):
        for mode in ("gather", "symmetric"):
            seed += 1
            out.append(dict(seed=seed, dim=dim, n=1600 if dim == 2 else 1728, nref=0, k=40, periodic=[False] * dim,
                            mode=mode, lattice=True))
    return out


def inputs_of(c):
    x, hx, y, hy, lo, hi, per = f64_case(c["seed"], c["dim"], c["n"], c["nref"], c["k"], c["periodic"], c["lattice"])
    return x, hx, y, hy, lo, hi, per
