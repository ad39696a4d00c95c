"""Serving: neighbour searches of many persistent scenes, continuously batched on one GPU.

A scene is a point cloud that lives on the device across requests -- one simulation or one
training scene whose points move a little between timesteps.  A request advances a scene (adds a
displacement to its points) and asks for its adjacency.  The server

* keeps every scene in a device arena (one per dimension: positions, supports, user indices and
  linear cells of all scenes in fixed segments), in the cell order of the scene's last search, so
  the next search re-sorts incrementally: only the points that changed cell are sorted and merged
  (``tcr_batch_desc.ref_lin_hint``) instead of rebuilding from scratch;
* admits pending requests in arrival order while their estimated device memory fits the HBM
  budget and their scene has no request in flight (a scene's requests run in order);
* admits pending requests in arrival order while the device bytes their searches need -- the
  structure and scratch sizes ``tcr_batch_sizes`` reports for the scene, its staging list and its
  output at the pair count of its last search -- fit the HBM budget, and their scene has no
  request waiting to be enqueued (a scene's requests run in order);
* enqueues each admitted group as one batched search (``tcr_batch_*``: one set of launches for
  all its scenes) on one of ``slots`` worker streams and does not wait for it: the worker goes
  straight back to admission, so groups are enqueued while earlier ones run (continuous
  batching).  A completion thread waits for each group's event, slices the per-scene results with
  offsets the device copied to pinned memory, and completes the requests; nothing on the worker
  reads device memory.  A scene's next request waits on the stream for its previous search's
  arena update (an event), not on the host.  The host work of a group is a fixed number of
  vectorised operations over the arena, whatever the number of scenes in it.

Results are in the scene's user numbering (``SparseCOO`` rows and columns are the indices the
scene was given with; rows come grouped in the scene's cell order), ready for use on the default
stream when the request completes, and a request's result does not depend on what it was batched
with: the batched engine gives each cloud exactly its single-search result.  The reference has no
serving layer; each request there is one ``radiusSearch`` call (src/torchCompactRadius/
neighborhood.py:136-309) that rebuilds its structure.
"""
import collections
import threading
import time
from typing import Dict, List, Optional

import numpy as np
import torch

import queue

from . import _lib
from . import context as _context
from .batched import batch_desc, cloud_table, enqueue_batch
from .search import _as_f32, _domain_host, _require_cuda
from .util import DomainDescription, SparseCOO

# Device bytes of a search beyond the library's structure and scratch: per point the arena
# indices of the group (int64 slot, shift), the user ids, the cell hint and the new cell order
# (int32 each); per staging word 4 bytes; per pair two int64 (COO row and column).
WORK_BYTES_PER_POINT = 32
STAGE_WORDS_PER_POINT = 24  # dense 3D clouds (50 neighbours) stage about 15 record words per point


class Scene:
    """What a scene starts from: positions [n, dim], supports [n], its domain and hashMapLength."""

    def __init__(self, positions: torch.Tensor, supports: torch.Tensor, domain: DomainDescription,
                 hashMapLength: int = 4096, expected_neighbours: float = 64.0):
        if positions.dim() != 2 or not 1 <= positions.shape[1] <= 3:
            raise ValueError("positions must be [n, dim] with dim 1, 2 or 3")
        if supports.shape[0] != positions.shape[0]:
            raise ValueError("one support per point")
        self.positions = positions
        self.supports = supports
        self.dim = int(positions.shape[1])
        self.n = int(positions.shape[0])
        self.lo, self.hi, self.mask = _domain_host(domain, self.dim)
        self.hashMapLength = int(hashMapLength)
        self.expected_neighbours = float(expected_neighbours)
        self.pairs = self.n * self.expected_neighbours  # pair count of the last search (estimate before one)
        self._lib_bytes = None

    def library_bytes(self) -> int:
        """Structure + scratch bytes of this scene's search with the incremental re-sort, as
        ``tcr_batch_sizes`` reports them (host-only; no device work)."""
        if self._lib_bytes is None:
            t = cloud_table(1)
            t["dim"][0] = self.dim
            t["n_query"][0] = t["n_ref"][0] = self.n
            hint = _FakePtr()  # a hint enlarges the scratch; sizing reads no pointer
            b = batch_desc(t, "gather", True, lin_hint=hint)
            s, w = _lib.batch_sizes(b)
            self._lib_bytes = int(s + w)
        return self._lib_bytes

    def bytes_estimate(self) -> int:
        """Device bytes one search of this scene needs: library structure and scratch, work arrays,
        staging list and COO output at the last search's pair count (plus 10%)."""
        return int(self.library_bytes() + self.n * (WORK_BYTES_PER_POINT + 4 * STAGE_WORDS_PER_POINT)
                   + 16 * 1.1 * self.pairs + 65536)


class _FakePtr:
    """Stands in for a device tensor in a descriptor that is only sized (data_ptr is never read)."""

    @staticmethod
    def data_ptr():
        return 256


class Request:
    """Advance scene `scene` by `displacement` (user order [n, dim], or None) -- or by Gaussian
    noise of standard deviation `jitter` drawn on the device -- and search it."""

    def __init__(self, scene: int, displacement: Optional[torch.Tensor] = None, arrival: Optional[float] = None,
                 jitter: Optional[float] = None, on_done=None):
        self.scene = scene
        self.displacement = displacement
        self.jitter = jitter
        self.on_done = on_done  # called by the worker with the request when it completes
        self.arrival = time.perf_counter() if arrival is None else arrival
        self.admitted = None
        self.finish = None
        self.result: Optional[SparseCOO] = None
        self.error: Optional[BaseException] = None
        self._done = threading.Event()

    def wait(self, timeout=None) -> SparseCOO:
        if not self._done.wait(timeout):
            raise TimeoutError("request not finished")
        if self.error is not None:
            raise self.error
        return self.result

    @property
    def latency(self):
        return None if self.finish is None else self.finish - self.arrival


class _Arena:
    """The scenes of one dimension on the device, each in a fixed segment."""

    def __init__(self, dim, scenes, device):
        self.dim = dim
        n = np.array([s.n for s in scenes], dtype=np.int64)
        self.base = np.zeros(len(scenes) + 1, dtype=np.int64)
        np.cumsum(n, out=self.base[1:])
        total = int(self.base[-1])
        self.pos = torch.empty(max(total, 1), dim, dtype=torch.float32, device=device)
        self.sup = torch.empty(max(total, 1), dtype=torch.float32, device=device)
        self.ids = torch.empty(max(total, 1), dtype=torch.int32, device=device)
        self.lin = torch.full((max(total, 1),), -1, dtype=torch.int32, device=device)  # no hint yet
        for k, s in enumerate(scenes):
            a, b = int(self.base[k]), int(self.base[k + 1])
            self.pos[a:b] = _as_f32(s.positions, device)
            self.sup[a:b] = _as_f32(s.supports, device)
            self.ids[a:b] = torch.arange(s.n, dtype=torch.int32, device=device)


class SearchServer:
    """Continuous-batching search server over persistent scenes (see the module docstring)."""

    def __init__(self, device=None, mode: str = "gather", hbm_budget: float = 40e9, slots: int = 2,
                 max_batch: int = 64):
        dev = _require_cuda(torch.device(device) if device is not None else torch.device("cuda"))
        self.device = dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.mode = mode
        self.hbm_budget = float(hbm_budget)
        self.slots = int(slots)
        self.max_batch = int(max_batch)
        self.scenes: List[Scene] = []
        self._arenas: Dict[int, _Arena] = {}
        self._tables = {}
        self._where = []  # scene -> (dim, index within its arena)
        self._pending = collections.deque()
        self._busy = set()
        self._in_use = 0
        self._cv = threading.Condition()
        self._running = False
        self._threads = []
        self._completer = None
        self._done = queue.Queue()
        self._last_event = {}  # scene -> event after the arena update of its last enqueued search
        self.batches = 0
        self.batched_requests = 0
        self.tuning = (0, 0)  # (queries per unit, walk blocks per SM) of the workers' searches; 0: default

    def set_tuning(self, config):
        """Tuning of the searches the workers make from now on (an Autotuner's `apply`)."""
        self.tuning = (int(config[0]), int(config[1]))

    # -- setup ----------------------------------------------------------------------------
    def add_scene(self, scene: Scene) -> int:
        """Adds a scene (before start())."""
        if self._running:
            raise RuntimeError("add scenes before starting the server")
        if scene.bytes_estimate() > self.hbm_budget:
            raise ValueError("the scene alone exceeds the HBM budget")
        self.scenes.append(scene)
        return len(self.scenes) - 1

    def _build_arenas(self):
        self._where = [None] * len(self.scenes)
        self._arenas, self._tables = {}, {}
        for dim in (1, 2, 3):
            ks = [k for k, s in enumerate(self.scenes) if s.dim == dim]
            if not ks:
                continue
            ar = _Arena(dim, [self.scenes[k] for k in ks], self.device)
            t = cloud_table(len(ks))
            for j, k in enumerate(ks):
                s = self.scenes[k]
                self._where[k] = (dim, j)
                t["dim"][j] = dim
                t["periodic_mask"][j] = s.mask
                t["domain_min"][j, :dim] = s.lo
                t["domain_max"][j, :dim] = s.hi
                t["hash_map_length"][j] = s.hashMapLength
                t["n_query"][j] = t["n_ref"][j] = s.n
                a = int(ar.base[j])
                t["query_pos"][j] = t["ref_pos"][j] = ar.pos.data_ptr() + 4 * dim * a
                t["query_sup"][j] = t["ref_sup"][j] = ar.sup.data_ptr() + 4 * a
            self._arenas[dim] = ar
            self._tables[dim] = t
        torch.cuda.synchronize(self.device)

    def positions(self, scene: int) -> torch.Tensor:
        """A scene's current positions in user order (call while it has no request in flight)."""
        if not self._where:
            return self.scenes[scene].positions
        ev = self._last_event.get(scene)
        if ev is not None:
            ev.synchronize()
        dim, j = self._where[scene]
        ar = self._arenas[dim]
        a, b = int(ar.base[j]), int(ar.base[j + 1])
        out = torch.empty_like(ar.pos[a:b])
        out.index_copy_(0, ar.ids[a:b].long(), ar.pos[a:b])
        return out

    def start(self):
        with self._cv:
            if self._running:
                return self
            self._build_arenas()
            self._running = True
        self._completer = threading.Thread(target=self._complete, daemon=True)
        self._completer.start()
        for slot in range(self.slots):
            t = threading.Thread(target=self._worker, args=(slot,), daemon=True)
            t.start()
            self._threads.append(t)
        return self

    def stop(self):
        with self._cv:
            self._running = False
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        self._threads = []
        if self._completer is not None:
            self._done.put(None)  # after every enqueued group
            self._completer.join()
            self._completer = None

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    # -- requests -------------------------------------------------------------------------
    def submit(self, request: Request) -> Request:
        if not 0 <= request.scene < len(self.scenes):
            raise IndexError(f"no scene {request.scene}")
        with self._cv:
            self._pending.append(request)
            self._cv.notify()
        return request

    def _admit(self):
        """Pending requests, in arrival order, whose scene is free and whose memory fits."""
        batch, scenes, blocked = [], set(), set()
        keep = collections.deque()
        while self._pending:
            r = self._pending.popleft()
            sc = self.scenes[r.scene]
            need = sc.bytes_estimate()
            if (r.scene in self._busy or r.scene in scenes or r.scene in blocked or len(batch) >= self.max_batch
                    or self._in_use + need > self.hbm_budget):
                keep.append(r)
                blocked.add(r.scene)  # later requests of the scene wait behind this one
                continue
            r._bytes = need
            batch.append(r)
            scenes.add(r.scene)
            self._in_use += need
        keep.extend(self._pending)
        self._pending = keep
        self._busy |= scenes
        return batch

    def _fail(self, reqs, ex):
        with self._cv:
            for r in reqs:
                self._in_use -= getattr(r, "_bytes", 0)
                r.error = ex
                r.finish = time.perf_counter()
            self._cv.notify_all()
        for r in reqs:
            r._done.set()

    def _worker(self, slot):
        try:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(self.device)
            ctx = _context.SearchContext()  # this worker's staging estimate
        except BaseException as ex:  # no worker: fail what waits instead of leaving it hanging
            with self._cv:
                reqs = list(self._pending)
                self._pending.clear()
            self._fail(reqs, ex)
            return
        while True:
            with self._cv:
                batch = []
                while self._running:
                    batch = self._admit()
                    if batch:
                        break
                    self._cv.wait(0.05)
                if not batch:
                    return
            launched = []
            try:
                ctx.unit_queries, ctx.walk_blocks_per_sm = self.tuning
                with _context.use(ctx):
                    for dim in (1, 2, 3):
                        group = [r for r in batch if self.scenes[r.scene].dim == dim]
                        if group:
                            self._done.put(self._launch(group, dim, stream, ctx))
                            launched += group
            except BaseException as ex:  # the requests report it; the server keeps serving
                self._fail([r for r in batch if r not in launched], ex)
            finally:
                # the scenes' next requests may be enqueued now: their device work waits for this
                # group's arena update on the stream (_last_event), not on the host
                with self._cv:
                    for r in batch:
                        self._busy.discard(r.scene)
                    self._cv.notify_all()

    def _launch(self, group, dim, stream, ctx):
        """Enqueues one batched search over the scenes of `group` (all of dimension dim) and the
        arena update after it; returns what the completion thread needs."""
        dev = self.device
        ar = self._arenas[dim]
        now = time.perf_counter()
        for r in group:
            r.admitted = now
        js = np.array([self._where[r.scene][1] for r in group], dtype=np.int64)
        n = ar.base[js + 1] - ar.base[js]
        bb = np.zeros(len(js) + 1, dtype=np.int64)  # batch bases
        np.cumsum(n, out=bb[1:])
        T = int(bb[-1])
        table = np.ascontiguousarray(self._tables[dim][js])
        user = torch.cuda.default_stream(dev)
        stream.wait_stream(user)  # explicit displacements made on the caller's stream are ready
        for r in group:
            ev = self._last_event.get(r.scene)
            if ev is not None:
                stream.wait_event(ev)  # the scene's previous search has updated its arena segment
        jit = np.array([r.jitter or 0.0 for r in group], dtype=np.float32)
        # the group's per-scene values in one pinned block, copied without waiting for the stream
        # (a copy from pageable memory would wait for the stream's earlier groups)
        host = torch.from_numpy(np.concatenate([n, ar.base[js] - bb[:-1], bb, jit.view(np.int32).astype(np.int64)]))
        host = host.pin_memory()
        G = len(group)
        with torch.cuda.stream(stream):
            vals = host.to(dev, non_blocking=True)
            ns, base_shift, bb_dev = vals[:G], vals[G:2 * G], vals[2 * G:3 * G + 1]
            # arena index of every batch slot: arena base of its scene + its offset in the scene
            # (expanded from per-scene values on the device)
            shift = torch.repeat_interleave(base_shift, ns, output_size=T)
            dst = torch.arange(T, device=dev) + shift
            if jit.any():
                sig = torch.repeat_interleave(vals[3 * G + 1:].to(torch.int32).view(torch.float32), ns, output_size=T)
                ar.pos.index_add_(0, dst, torch.randn(T, dim, device=dev) * sig[:, None])
            for k, r in enumerate(group):
                if r.displacement is not None:
                    a, b = int(ar.base[js[k]]), int(ar.base[js[k] + 1])
                    d = r.displacement.to(device=dev, dtype=torch.float32, non_blocking=True)
                    ar.pos[a:b] += d.index_select(0, ar.ids[a:b].long())
            ids = ar.ids.index_select(0, dst)
            hint = ar.lin.index_select(0, dst)
            lin_out = torch.empty(T, dtype=torch.int32, device=dev)
            order_out = torch.empty(T, dtype=torch.int32, device=dev)
            cap = int(1.1 * sum(self.scenes[r.scene].pairs for r in group)) + 4096
            stage_cap = int(ctx.batch_stage_per_query * 1.1 * T) + 65536
            pend = enqueue_batch(table, self.mode, True, "coo", dev, stream, cap, stage_cap, local_index=False,
                                 query_ids=ids, ref_ids=ids, lin_hint=hint, lin_out=lin_out, order_out=order_out,
                                 base_index=bb_dev)
            # keep every scene in its new cell order (the next search re-sorts incrementally)
            src = order_out.long() + shift
            ar.pos.index_copy_(0, dst, ar.pos.index_select(0, src))
            ar.sup.index_copy_(0, dst, ar.sup.index_select(0, src))
            ar.ids.index_copy_(0, dst, ar.ids.index_select(0, src))
            ar.lin.index_copy_(0, dst, lin_out)
            ev = torch.cuda.Event()
            ev.record(stream)
        for r in group:
            self._last_event[r.scene] = ev
        pend.keep = (host, vals, shift, dst, ids, hint, lin_out, order_out, src)
        return group, n, pend, ctx

    def _complete(self):
        """Waits for each enqueued group in order and completes its requests."""
        user = torch.cuda.default_stream(self.device)
        while True:
            item = self._done.get()
            if item is None:
                return
            group, n, pend, ctx = item
            try:
                total = pend.finish()
                offs = pend.offsets_host.tolist()
                for t in (pend.row, pend.col):
                    t.record_stream(user)  # results are read on the default stream
                for k, r in enumerate(group):
                    m = int(n[k])
                    a, b = offs[k], offs[k + 1]
                    r.result = SparseCOO(pend.row[a:b], pend.col[a:b], m, m)
                    self.scenes[r.scene].pairs = b - a
                if len(n):
                    ctx.batch_stage_per_query = max(int(pend.info[4]) / max(int(n.sum()), 1), 1.0)
                del total
            except BaseException as ex:  # the requests report it; the server keeps serving
                for r in group:
                    r.error = ex
            now = time.perf_counter()
            with self._cv:
                for r in group:
                    self._in_use -= getattr(r, "_bytes", 0)
                    r.finish = now
                self.batches += 1
                self.batched_requests += len(group)
                self._cv.notify_all()
            for r in group:
                if r.on_done is not None:
                    try:
                        r.on_done(r)
                    except BaseException as ex:
                        r.error = ex
                r._done.set()

    # -- convenience ----------------------------------------------------------------------
    def search(self, scene: int, displacement: Optional[torch.Tensor] = None, timeout=None,
               jitter: Optional[float] = None) -> SparseCOO:
        """Submits one request and waits for it."""
        return self.submit(Request(scene, displacement, jitter=jitter)).wait(timeout)
