"""Serving: neighbour searches of many persistent scenes, continuously batched on one GPU.

A scene is a point cloud that lives on the device across requests -- one simulation or one
training scene whose points move a little between timesteps.  A request advances a scene (adds a
displacement to its points) and asks for its adjacency.  The server

* keeps every scene on the device in the cell order of its last search, with each point's user
  index and linear cell: the next search of the scene re-sorts incrementally (only the points
  that changed cell are sorted and merged, ``tcr_batch_desc.ref_lin_hint``) instead of
  rebuilding from scratch;
* admits pending requests in arrival order while their estimated device memory fits the HBM
  budget and their scene has no request in flight (a scene's requests run in order);
* runs each admitted group as one batched search (``tcr_batch_*``: one set of launches for all
  its scenes) on one of ``slots`` worker streams, so a group admitted while another is still on
  the GPU runs beside it: requests that arrive during a search are admitted as soon as a slot and
  memory free up (continuous batching), not after the queue drains.

Results are in the scene's user numbering (``SparseCOO`` rows and columns are the indices the
scene was created with; rows come grouped in the scene's cell order), ready for use on the default
stream when the request completes, and a request's result does not depend on what it was batched
with: the batched engine gives each cloud exactly its single-search result.  The reference has no serving
layer; each request there is one ``radiusSearch`` call (src/torchCompactRadius/neighborhood.py:
136-309) that rebuilds its structure.
"""
import collections
import threading
import time
from typing import List, Optional

import numpy as np
import torch

from .batched import BatchBuffers, cloud_table, run_batch
from .search import _as_f32, _domain_host, _require_cuda
from .util import DomainDescription, SparseCOO

# Device bytes one search needs per point and per expected pair (structure, scratch with the
# incremental re-sort, staging list and int64 COO output), for admission.
BYTES_PER_POINT = 420
BYTES_PER_PAIR = 22


class Scene:
    """A persistent cloud on the device, stored in the cell order of its last search."""

    def __init__(self, positions: torch.Tensor, supports: torch.Tensor, domain: DomainDescription,
                 hashMapLength: int = 4096, device=None, expected_neighbours: float = 64.0):
        device = _require_cuda(torch.device(device) if device is not None else positions.device)
        self.device = device
        self.dim = int(positions.shape[1])
        self.n = int(positions.shape[0])
        self.pos = _as_f32(positions, device).clone()          # stored order
        self.sup = _as_f32(supports, device).clone()
        self.ids = torch.arange(self.n, dtype=torch.int32, device=device)  # user index of stored point k
        self.lin = None                                        # linear cell of stored point k (the hint)
        self.lo, self.hi, self.mask = _domain_host(domain, self.dim)
        self.hashMapLength = int(hashMapLength)
        self.expected_neighbours = float(expected_neighbours)
        self.steps = 0

    def positions(self) -> torch.Tensor:
        """Current positions in user order."""
        out = torch.empty_like(self.pos)
        out.index_copy_(0, self.ids.long(), self.pos)
        return out

    def supports(self) -> torch.Tensor:
        out = torch.empty_like(self.sup)
        out.index_copy_(0, self.ids.long(), self.sup)
        return out

    def bytes_estimate(self) -> int:
        return int(self.n * (BYTES_PER_POINT + BYTES_PER_PAIR * self.expected_neighbours))


class Request:
    """Advance scene `scene` by `displacement` (user order [n, dim], or None) -- or by Gaussian
    noise of standard deviation `jitter` drawn on the device from `seed` -- and search it."""

    def __init__(self, scene: int, displacement: Optional[torch.Tensor] = None, arrival: Optional[float] = None,
                 jitter: Optional[float] = None, seed: Optional[int] = None, on_done=None):
        self.scene = scene
        self.on_done = on_done  # called by the worker with the request when it completes
        self.displacement = displacement
        self.jitter = jitter  # instead of a displacement: N(0, jitter^2) per coordinate, drawn on the device
        self.seed = seed
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
        self._pending = collections.deque()
        self._busy = set()
        self._in_use = 0
        self._cv = threading.Condition()
        self._running = False
        self._threads = []
        self.batches = 0
        self.batched_requests = 0

    # -- setup ----------------------------------------------------------------------------
    def add_scene(self, scene: Scene) -> int:
        if scene.bytes_estimate() > self.hbm_budget:
            raise ValueError("the scene alone exceeds the HBM budget")
        self.scenes.append(scene)
        return len(self.scenes) - 1

    def start(self):
        with self._cv:
            if self._running:
                return self
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
            bufs = BatchBuffers(self.device)
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
                self._run(batch, stream, bufs)
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

    def _run(self, batch, stream, bufs):
        dev = self.device
        for r in batch:
            r.admitted = time.perf_counter()
        scenes = [self.scenes[r.scene] for r in batch]
        user = torch.cuda.default_stream(dev)
        stream.wait_stream(user)  # displacements and scenes made on the caller's stream are ready
        for sc in scenes:  # scene arrays move between worker streams: no reuse before this one is done
            for t in (sc.pos, sc.sup, sc.ids, sc.lin):
                if t is not None:
                    t.record_stream(stream)
        with torch.cuda.stream(stream):
            for r, sc in zip(batch, scenes):
                if r.displacement is not None:
                    d = r.displacement.to(device=dev, dtype=torch.float32, non_blocking=True)
                    sc.pos.add_(d.index_select(0, sc.ids.long()))
                elif r.jitter:
                    g = torch.Generator(device=dev)
                    g.manual_seed(int(r.seed) if r.seed is not None else int(time.perf_counter_ns()))
                    d = torch.randn(sc.pos.shape, generator=g, device=dev) * float(r.jitter)
                    sc.pos.add_(d.index_select(0, sc.ids.long()))
            C = len(scenes)
            table = cloud_table(C)
            n = np.array([sc.n for sc in scenes], dtype=np.int64)
            base = np.zeros(C + 1, dtype=np.int64)
            np.cumsum(n, out=base[1:])
            for k, sc in enumerate(scenes):
                table["dim"][k] = sc.dim
                table["periodic_mask"][k] = sc.mask
                table["domain_min"][k, :sc.dim] = sc.lo
                table["domain_max"][k, :sc.dim] = sc.hi
                table["hash_map_length"][k] = sc.hashMapLength
                table["n_query"][k] = table["n_ref"][k] = sc.n
                table["query_pos"][k] = table["ref_pos"][k] = sc.pos.data_ptr() if sc.n else 0
                table["query_sup"][k] = table["ref_sup"][k] = sc.sup.data_ptr() if sc.n else 0
            total = int(base[-1])
            ids = torch.cat([sc.ids for sc in scenes]) if C > 1 else scenes[0].ids
            hint = None
            if any(sc.lin is not None for sc in scenes):
                hint = torch.cat([sc.lin if sc.lin is not None else
                                  torch.full((sc.n,), -1, dtype=torch.int32, device=dev) for sc in scenes])
            lin_out = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
            order_out = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
            out = run_batch(table, self.mode, True, "coo", dev, local_index=False, query_ids=ids, ref_ids=ids,
                            buffers=bufs, stream=stream, lin_hint=hint, lin_out=lin_out, order_out=order_out,
                            fresh_outputs=True)
            for t in (out["row"], out["col"]):
                t.record_stream(user)  # results are read on the default stream
            offs = out["offsets"].index_select(0, torch.as_tensor(base, device=dev)).cpu().tolist()
            for k, (r, sc) in enumerate(zip(batch, scenes)):
                p0, p1 = offs[k], offs[k + 1]
                r.result = SparseCOO(out["row"][p0:p1], out["col"][p0:p1], sc.n, sc.n)
                # keep the scene in its new cell order: the next search re-sorts incrementally
                perm = (order_out[int(base[k]):int(base[k + 1])] - int(base[k])).long()
                sc.pos = sc.pos.index_select(0, perm)
                sc.sup = sc.sup.index_select(0, perm)
                sc.ids = sc.ids.index_select(0, perm)
                sc.lin = lin_out[int(base[k]):int(base[k + 1])].clone()
                sc.steps += 1
            stream.synchronize()

    # -- convenience ----------------------------------------------------------------------
    def search(self, scene: int, displacement: Optional[torch.Tensor] = None, timeout=None) -> SparseCOO:
        """Submits one request and waits for it."""
        return self.submit(Request(scene, displacement)).wait(timeout)
