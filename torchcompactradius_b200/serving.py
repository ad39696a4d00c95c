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
* runs each admitted group as one batched search (``tcr_batch_*``: one set of launches for all
  its scenes) on one of ``slots`` worker streams, so a group admitted while another is still on
  the GPU runs beside it: requests that arrive during a search are admitted as soon as a slot and
  memory free up (continuous batching), not after the queue drains.  The host work of a group is
  a fixed number of vectorised operations over the arena, whatever the number of scenes in it.

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

from . import context as _context
from .batched import BatchBuffers, cloud_table, run_batch
from .search import _as_f32, _domain_host, _require_cuda
from .util import DomainDescription, SparseCOO

# Device bytes one search needs per point and per expected pair (structure, scratch with the
# incremental re-sort, staging list and int64 COO output), for admission.
BYTES_PER_POINT = 420
BYTES_PER_PAIR = 22


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

    def bytes_estimate(self) -> int:
        return int(self.n * (BYTES_PER_POINT + BYTES_PER_PAIR * self.expected_neighbours))


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
            batch.append(r)
            scenes.add(r.scene)
            self._in_use += need
        keep.extend(self._pending)
        self._pending = keep
        self._busy |= scenes
        return batch

    def _worker(self, slot):
        try:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(self.device)
            bufs = {d: BatchBuffers(self.device) for d in (1, 2, 3)}
            ctx = _context.SearchContext()  # this worker's size estimates
        except BaseException as ex:  # no worker: fail what waits instead of leaving it hanging
            with self._cv:
                while self._pending:
                    r = self._pending.popleft()
                    r.error = ex
                    r._done.set()
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
            try:
                ctx.unit_queries, ctx.walk_blocks_per_sm = self.tuning
                with _context.use(ctx):
                    for dim in (1, 2, 3):
                        group = [r for r in batch if self.scenes[r.scene].dim == dim]
                        if group:
                            self._run(group, dim, stream, bufs[dim])
            except BaseException as ex:  # the requests report it; the server keeps serving
                for r in batch:
                    r.error = ex
            finally:
                now = time.perf_counter()
                with self._cv:
                    for r in batch:
                        self._busy.discard(r.scene)
                        self._in_use -= self.scenes[r.scene].bytes_estimate()
                        r.finish = now
                    self.batches += 1
                    self.batched_requests += len(batch)
                    self._cv.notify_all()
                for r in batch:
                    if r.on_done is not None:
                        try:
                            r.on_done(r)
                        except BaseException as ex:
                            r.error = ex
                    r._done.set()

    def _run(self, group, dim, stream, bufs):
        """One batched search over the scenes of `group` (all of dimension dim)."""
        dev = self.device
        ar = self._arenas[dim]
        for r in group:
            r.admitted = time.perf_counter()
        js = np.array([self._where[r.scene][1] for r in group], dtype=np.int64)
        n = ar.base[js + 1] - ar.base[js]
        bb = np.zeros(len(js) + 1, dtype=np.int64)  # batch bases
        np.cumsum(n, out=bb[1:])
        T = int(bb[-1])
        table = np.ascontiguousarray(self._tables[dim][js])
        user = torch.cuda.default_stream(dev)
        stream.wait_stream(user)  # explicit displacements made on the caller's stream are ready
        with torch.cuda.stream(stream):
            # arena index of every batch slot: arena base of its scene + its offset in the scene
            # (expanded from per-scene values on the device)
            ns = torch.as_tensor(n, device=dev)
            shift = torch.repeat_interleave(torch.as_tensor(ar.base[js] - bb[:-1], device=dev), ns, output_size=T)
            dst = torch.arange(T, device=dev) + shift
            jit = np.array([r.jitter or 0.0 for r in group], dtype=np.float32)
            if jit.any():
                sig = torch.repeat_interleave(torch.as_tensor(jit, device=dev), ns, output_size=T)
                ar.pos.index_add_(0, dst, torch.randn(T, dim, device=dev) * sig[:, None])
            for k, r in enumerate(group):
                if r.displacement is not None:
                    a, b = int(ar.base[js[k]]), int(ar.base[js[k] + 1])
                    d = r.displacement.to(device=dev, dtype=torch.float32, non_blocking=True)
                    ar.pos[a:b] += d.index_select(0, ar.ids[a:b].long())
            ids = ar.ids.index_select(0, dst)
            hint = ar.lin.index_select(0, dst)
            lin_out = bufs.get("lin_out", T, torch.int32)
            order_out = bufs.get("order_out", T, torch.int32)
            out = run_batch(table, self.mode, True, "coo", dev, local_index=False, query_ids=ids, ref_ids=ids,
                            buffers=bufs, stream=stream, lin_hint=hint, lin_out=lin_out, order_out=order_out,
                            fresh_outputs=True)
            for t in (out["row"], out["col"]):
                t.record_stream(user)  # results are read on the default stream
            # keep every scene in its new cell order (the next search re-sorts incrementally)
            src = order_out.long() + shift
            ar.pos.index_copy_(0, dst, ar.pos.index_select(0, src))
            ar.sup.index_copy_(0, dst, ar.sup.index_select(0, src))
            ar.ids.index_copy_(0, dst, ar.ids.index_select(0, src))
            ar.lin.index_copy_(0, dst, lin_out)
            offs = out["offsets"].index_select(0, torch.as_tensor(bb, device=dev)).cpu().tolist()
            for k, r in enumerate(group):
                m = int(n[k])
                r.result = SparseCOO(out["row"][offs[k]:offs[k + 1]], out["col"][offs[k]:offs[k + 1]], m, m)
            stream.synchronize()

    # -- convenience ----------------------------------------------------------------------
    def search(self, scene: int, displacement: Optional[torch.Tensor] = None, timeout=None,
               jitter: Optional[float] = None) -> SparseCOO:
        """Submits one request and waits for it."""
        return self.submit(Request(scene, displacement, jitter=jitter)).wait(timeout)
