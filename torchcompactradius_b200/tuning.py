"""Autotuner for the walks' run-time parameters.

Two parameters of the engine change its speed and never its results (a query's candidates and
their order do not depend on them):

* queries per work unit -- 32, 16 or 8.  A unit is one warp; with fewer queries per unit each
  query gets 2 or 4 lanes (the candidate streams of the walk), which pays for sparse clouds whose
  cells hold few points and costs more stencil look-ups for dense ones;
* resident walk blocks per SM -- the size of the persistent walk grid.

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

_cache: Dict[Hashable, Config] = {}
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


class Autotuner:
    def __init__(self, candidates: Sequence[Config] = CANDIDATES, reps: int = 3):
        self.candidates = list(candidates)
        self.reps = int(reps)
        self.timings: Dict[Hashable, Dict[Config, float]] = {}

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
                run()
                ms = []
                for _ in range(self.reps):
                    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s.record(stream)
                    run()
                    e.record(stream)
                    e.synchronize()
                    ms.append(s.elapsed_time(e))
                times[cfg] = statistics.median(ms)
        best = min(times, key=times.get)
        (apply or (lambda cfg: set_tuning(*cfg, ctx=home)))(best)
        with _lock:
            if key is not None:
                _cache[key] = best
                self.timings[key] = times
        self.last_timings = times
        return best
