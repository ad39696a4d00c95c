"""Autotuner for the walks' run-time parameters.

Two parameters of the engine change its speed and never its results (a query's candidates and
their order do not depend on them):

* queries per work unit -- 32, 16 or 8.  A unit is one warp; with fewer queries per unit each
  query gets 2 or 4 lanes (the candidate streams of the walk), which pays for sparse clouds whose
  cells hold few points and costs more stencil look-ups for dense ones;
* resident walk blocks per SM -- the size of the persistent walk grid;
* the cell-size multiplier of single searches (``cell_scales``): cells m times the largest
  threshold on the exact clamped grid, which pays for sparse clouds whose reference-size cells hold
  few points.  Its pair set is the reference's whenever every point lies inside the domain on its
  non-periodic dimensions; the tuner keeps a multiplier only if it reproduced the pair set of the
  reference-size cells on the tuning run.

``Autotuner.tune(run, key)`` times every candidate setting on the caller's own search (``run`` is
a callable that performs one search on the current stream), leaves the fastest in the caller's
current ``SearchContext`` (``context.py``: per thread, or the one made current by
``context.use``) and remembers it under ``key`` (for example ``signature(...)`` of the workload),
so a later call with the same key sets it without timing.  Settings travel to the engine in each
search's descriptor, so tuning on one thread never changes another thread's searches.  The
reference has nothing to tune: its kernels use one thread per query.
"""
import statistics
import threading
from typing import Callable, Dict, Hashable, List, Optional, Sequence, Tuple

import torch

from . import context as _context

Config = Tuple[int, int]  # (queries per unit, walk blocks per SM)
DEFAULT: Config = (32, 12)
CANDIDATES: List[Config] = [(32, 12), (16, 12), (8, 12), (32, 8), (16, 8), (32, 16), (16, 16)]

CELL_SCALES: Tuple[float, ...] = (1.0, 1.25, 1.5, 2.0)

_cache: Dict[Hashable, Config] = {}
_scale_cache: Dict[Hashable, float] = {}
_lock = threading.Lock()


def set_tuning(unit_queries: int = 0, walk_blocks_per_sm: int = 0, ctx: Optional[_context.SearchContext] = None):
    """Sets the tuning of later searches in ``ctx`` (default: this thread's current context); 0
    keeps a default.  The engine checks the values when a search is made."""
    if unit_queries not in (0, 8, 16, 32):
        raise ValueError("unit_queries must be 8, 16 or 32 (0: default 32)")
    if not 0 <= walk_blocks_per_sm <= 64:
        raise ValueError("walk_blocks_per_sm must be in [1, 64] (0: default 12)")
    ctx = ctx or _context.current()
    ctx.unit_queries, ctx.walk_blocks_per_sm = int(unit_queries), int(walk_blocks_per_sm)


def signature(dims: Sequence[int], periodic: Sequence[bool], n_points: int, mode: str, neighbours: float) -> Hashable:
    """A workload key: dimensions and periodicity present, mode, and the sizes rounded to powers
    of two (tuning carries over between workloads of the same shape)."""
    import math
    return (tuple(sorted(set(int(d) for d in dims))), tuple(sorted(set(bool(p) for p in periodic))), mode,
            int(math.log2(max(n_points, 1))), int(math.log2(max(neighbours, 1.0))))


def same_pairs(a, b) -> bool:
    """Whether two search results (SparseCSR or SparseCOO) hold the same pairs per row, whatever
    the order within a row."""
    def keys(r):
        if hasattr(r, "indptr"):
            counts = torch.diff(r.indptr.to(torch.int64))
            row = torch.repeat_interleave(torch.arange(counts.numel(), device=counts.device), counts)
            col = r.indices
        else:
            row, col = r.row, r.col
        return torch.sort(row.to(torch.int64) * (1 << 32) + col.to(torch.int64)).values
    ka, kb = keys(a), keys(b)
    return ka.numel() == kb.numel() and bool(torch.equal(ka, kb))


class Autotuner:
    def __init__(self, candidates: Sequence[Config] = CANDIDATES, reps: int = 3):
        self.candidates = list(candidates)
        self.reps = int(reps)
        self.timings: Dict[Hashable, Dict[Config, float]] = {}
        self.scale_timings: Dict[Hashable, Dict[float, float]] = {}

    def _time(self, run, stream):
        run()
        ms = []
        for _ in range(self.reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            run()
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
        return statistics.median(ms)

    def tune_cell_scale(self, run: Callable[[], object], key: Optional[Hashable] = None,
                        scales: Sequence[float] = CELL_SCALES) -> float:
        """Times `run` (a single search returning its adjacency) at every cell-size multiplier in
        the current context's tuning, keeps the fastest whose pair set equals the one with
        reference-size cells, and leaves it in the current context; a key seen before only sets its
        remembered multiplier."""
        home = _context.current()
        with _lock:
            if key is not None and key in _scale_cache:
                home.cell_scale = _scale_cache[key]
                return home.cell_scale
        stream = torch.cuda.current_stream()
        trial = home.copy()
        times: Dict[float, float] = {}
        with _context.use(trial):
            trial.cell_scale = 1.0
            ref = run()
            for m in scales:
                trial.cell_scale = float(m)
                if m != 1.0 and not same_pairs(ref, run()):
                    continue  # a point outside the domain: this multiplier changes the pair set
                times[float(m)] = self._time(run, stream)
        best = min(times, key=times.get)
        home.cell_scale = best
        with _lock:
            if key is not None:
                _scale_cache[key] = best
                self.scale_timings[key] = times
        return best

    def tune(self, run: Callable[[], object], key: Optional[Hashable] = None,
             apply: Optional[Callable[[Config], None]] = None) -> Config:
        """Times `run` under every candidate setting (median of `reps` after one warm-up) and
        leaves the fastest in force; a key seen before only sets its remembered setting.  By
        default a setting is put in force in the current context, and `run` is timed inside a
        private copy of it, so the caller's size estimates and tuning change only by the final
        choice; `apply(config)` replaces that for searches made elsewhere (for example by a
        server's worker threads: ``SearchServer.set_tuning``)."""
        home = _context.current()
        trial = home.copy()
        put = apply or (lambda cfg: set_tuning(*cfg, ctx=trial))
        with _lock:
            if key is not None and key in _cache:
                (apply or (lambda cfg: set_tuning(*cfg, ctx=home)))(_cache[key])
                return _cache[key]
        stream = torch.cuda.current_stream()
        times: Dict[Config, float] = {}
        with _context.use(trial):
            for cfg in self.candidates:
                put(cfg)
                times[cfg] = self._time(run, stream)
        best = min(times, key=times.get)
        (apply or (lambda cfg: set_tuning(*cfg, ctx=home)))(best)
        with _lock:
            if key is not None:
                _cache[key] = best
                self.timings[key] = times
        self.last_timings = times
        return best
