"""Per-caller state of the searches: the tuning they run with and the sizes they learn.

A ``SearchContext`` holds what one caller's searches share and no other caller sees:

* the tuning -- queries per work unit of the walks (32, 16 or 8) and resident walk blocks per SM
  (0 keeps the engine's default), which travel to the engine in each call's descriptor
  (``tcr_search_desc`` / ``tcr_batch_desc``), so the engine keeps no tuning state; and the cell-size
  multiplier of single searches (1: the reference's cell; m > 1: cells m times the largest
  threshold on the exact clamped grid -- the same pair set whenever every point lies inside the
  domain on its non-periodic dimensions).  None of them changes such a result;
* the output and staging-list sizes per query learnt from the previous search, which size the
  buffers of the next one (a short estimate costs a second emit, never a wrong result).

Every thread has its own default context; ``use(ctx)`` makes ``ctx`` the current context of this
thread inside a ``with`` block, so a server worker, a captured plan or an autotuner that times
candidate settings never sees another caller's state.
"""
import contextlib
import copy
import threading
from dataclasses import dataclass


@dataclass
class SearchContext:
    unit_queries: int = 0        # queries per work unit: 32, 16 or 8 (0: default 32)
    walk_blocks_per_sm: int = 0  # resident walk blocks per SM, 1..64 (0: default 12)
    cell_scale: float = 1.0      # cell-size multiplier of single searches (1: the reference's cell)
    pairs_per_query: float = 64.0        # single searches: output pairs per query last time
    stage_per_query: float = 64.0        # single searches: staging words per query last time
    batch_pairs_per_query: float = 64.0  # batched searches
    batch_stage_per_query: float = 64.0
    level_stage_per_query: float = 96.0  # multi-level searches: staging words per level-pair query

    def copy(self) -> "SearchContext":
        return copy.copy(self)

    def tuning(self):
        return int(self.unit_queries), int(self.walk_blocks_per_sm)


_tls = threading.local()


def current() -> SearchContext:
    """The current context of this thread (its default one unless inside ``use``)."""
    stack = getattr(_tls, "stack", None)
    if stack:
        return stack[-1]
    ctx = getattr(_tls, "default", None)
    if ctx is None:
        ctx = _tls.default = SearchContext()
    return ctx


@contextlib.contextmanager
def use(ctx: SearchContext):
    """Makes ``ctx`` the current context of this thread for the ``with`` block."""
    stack = getattr(_tls, "stack", None)
    if stack is None:
        stack = _tls.stack = []
    stack.append(ctx)
    try:
        yield ctx
    finally:
        stack.pop()


def apply_tuning(desc, ctx: SearchContext = None):
    """Copies the context's tuning into a search or batch descriptor."""
    ctx = ctx or current()
    desc.unit_queries, desc.walk_blocks_per_sm = ctx.tuning()
    return desc
