"""Autotuner for the walks' run-time parameters.

Two parameters of the engine change its speed and never its results (a query's candidates and
their order do not depend on them):

* queries per work unit -- 32, 16 or 8.  A unit is one warp; with fewer queries per unit each
  query gets 2 or 4 lanes (the candidate streams of the walk), which pays for sparse clouds whose
  cells hold few points and costs more stencil look-ups for dense ones;
* resident walk blocks per SM -- the size of the persistent walk grid.

``Autotuner.tune(run, key)`` times every candidate setting on the caller's own search (``run`` is
a callable that performs one search on the current stream), keeps the fastest with
``tcr_set_tuning`` and remembers it under ``key`` (for example ``signature(...)`` of the workload),
so a later call with the same key sets it without timing.  The reference has nothing to tune: its
kernels use one thread per query.
"""
import statistics
import threading
from typing import Callable, Dict, Hashable, List, Optional, Sequence, Tuple

import torch

from . import _lib

Config = Tuple[int, int]  # (queries per unit, walk blocks per SM)
DEFAULT: Config = (32, 12)
CANDIDATES: List[Config] = [(32, 12), (16, 12), (8, 12), (32, 8), (16, 8), (32, 16), (16, 16)]

_cache: Dict[Hashable, Config] = {}
_lock = threading.Lock()


def set_tuning(unit_queries: int = 0, walk_blocks_per_sm: int = 0):
    """Sets the engine's tuning for later searches of this process (0 keeps a default)."""
    _lib.check(_lib.load().tcr_set_tuning(int(unit_queries), int(walk_blocks_per_sm)), "tcr_set_tuning")


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

    def tune(self, run: Callable[[], object], key: Optional[Hashable] = None) -> Config:
        """Times `run` under every candidate setting (median of `reps` after one warm-up) and
        leaves the fastest in force; a key seen before only sets its remembered setting."""
        with _lock:
            if key is not None and key in _cache:
                set_tuning(*_cache[key])
                return _cache[key]
        stream = torch.cuda.current_stream()
        times: Dict[Config, float] = {}
        try:
            for cfg in self.candidates:
                set_tuning(*cfg)
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
        except BaseException:
            set_tuning(*DEFAULT)
            raise
        best = min(times, key=times.get)
        set_tuning(*best)
        with _lock:
            if key is not None:
                _cache[key] = best
                self.timings[key] = times
        self.last_timings = times
        return best
