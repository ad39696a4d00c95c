"""Searches recorded once as CUDA graphs and replayed.

A search (or a batch) whose sizes and buffers stay fixed -- the next timestep of a simulation,
the next step of a training loop -- repeats the same ~40 kernel launches and their host work.
``SearchPlan`` runs it once eagerly to size the staging list and the output, records the
``tcr_batch_build_structure`` / ``tcr_batch_count`` / ``tcr_batch_emit`` sequence into one CUDA
graph, and from then on launches that graph: one launch and one synchronisation (to read the pair
count) per search.  Inputs are read from device buffers the plan was built on; the caller refreshes
them in place between replays (``StaticSearch.update`` does that for one cloud).

Every kernel re-initialises what it reads (counters, sort state, map), so a replay is a complete
search.  A replay whose pairs exceed the recorded output capacity (points that moved into denser
configurations) emits again eagerly into larger buffers -- the count of the replay stays valid --
and the graph is recorded again for the next replay; units whose records do not fit the recorded
staging list are re-walked by the emit pass, so no capacity can make a result wrong.
"""
import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .batched import batch_desc, cloud_table
from .search import _as_f32, _check_device_fault, _domain_host, _ptr, _require_cuda
from .util import DomainDescription, PointCloud, SparseCOO, SparseCSR


class SearchPlan:
    """A batched search of fixed sizes over fixed input buffers, replayed as a CUDA graph.

    ``table`` is a cloud table (``batched.cloud_table``) whose pointers name device buffers that
    stay alive and keep their addresses; ``replay()`` returns the same dict as ``run_batch``."""

    def __init__(self, table, mode: str, self_search: bool, fmt: str, device=None, local_index: bool = True,
                 slack: float = 0.25, stream: Optional[torch.cuda.Stream] = None):
        dev = _require_cuda(torch.device(device) if device is not None else torch.device("cuda"))
        self.device = dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.table = np.ascontiguousarray(table)
        self.fmt = fmt
        self.slack = float(slack)
        self.desc = batch_desc(self.table, mode, self_search, local_index)
        self.lib = _lib.load()
        self.s_bytes, self.w_bytes = _lib.batch_sizes(self.desc)
        self.nq = int(self.table["n_query"].sum())
        self.stream = stream or torch.cuda.Stream(self.device)
        d = self.device
        self.structure = torch.empty(self.s_bytes, dtype=torch.uint8, device=d)
        self.scratch = torch.empty(self.w_bytes, dtype=torch.uint8, device=d)
        self.offsets = torch.empty(self.nq + 1, dtype=torch.int64, device=d)
        self.counts = torch.empty(max(self.nq, 1), dtype=torch.int64, device=d)
        self.indptr = torch.empty(self.nq + 1, dtype=torch.int32, device=d) if fmt == "csr" else None
        self.info = torch.zeros(8, dtype=torch.int64, pin_memory=True)
        # first run, eagerly, with generous buffers: it sizes the staging list and the output
        self.stage = torch.empty(int(min(0x7fffffff, 128 * self.nq + 65536)), dtype=torch.int32, device=d)
        self._alloc_out(int(min(0x7fffffff, 64 * self.nq + 4096)))
        self.stream.wait_stream(torch.cuda.current_stream(d))
        with torch.cuda.stream(self.stream):
            self._enqueue()
        self.stream.synchronize()
        self._check()
        total = int(self.info[0])
        words = int(self.info[4])
        if total > self.cap:
            self._alloc_out(self._grown(total))
            with torch.cuda.stream(self.stream):
                self._emit()
            self.stream.synchronize()
        self.stage = torch.empty(int(min(0x7fffffff, words * (1 + self.slack) + 65536)), dtype=torch.int32, device=d)
        self._alloc_out(self._grown(total))
        self.graph = None
        self._record()

    # -- internals ------------------------------------------------------------------------
    def _grown(self, total):
        return int(min(0x7fffffff, total * (1 + self.slack) + 4096))

    def _alloc_out(self, cap):
        self.cap = cap
        self.col = torch.empty(max(cap, 1), dtype=torch.int64, device=self.device)
        self.row = torch.empty(max(cap, 1), dtype=torch.int64, device=self.device) if self.fmt == "coo" else None

    def _sptr(self):
        return ctypes.c_void_p(self.stream.cuda_stream)

    def _emit(self):
        _lib.check(self.lib.tcr_batch_emit(ctypes.byref(self.desc), _ptr(self.structure), _ptr(self.scratch),
                                           self.w_bytes, _ptr(self.stage), _ptr(self.offsets), _ptr(self.row),
                                           _ptr(self.col), self.cap, self._sptr()), "tcr_batch_emit")

    def _enqueue(self):
        lib, sp = self.lib, self._sptr()
        _lib.check(lib.tcr_batch_build_structure(ctypes.byref(self.desc), _ptr(self.structure), self.s_bytes,
                                                 _ptr(self.scratch), self.w_bytes, sp), "tcr_batch_build_structure")
        _lib.check(lib.tcr_batch_count(ctypes.byref(self.desc), _ptr(self.structure), _ptr(self.scratch),
                                       self.w_bytes, _ptr(self.stage), self.stage.numel(), _ptr(self.offsets),
                                       _ptr(self.indptr), _ptr(self.counts), ctypes.c_void_p(self.info.data_ptr()),
                                       sp), "tcr_batch_count")
        self._emit()

    def _record(self):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            self._enqueue()
        self.graph = g

    def _check(self):
        _check_device_fault(self.info)
        if int(self.info[1]) != 0:
            raise ValueError(f"{int(self.info[1])} cloud(s) have no valid cell grid for their domain and support")

    # -- use ------------------------------------------------------------------------------
    def replay(self):
        """One search through the recorded graph; returns the outputs (views into the plan's
        buffers, valid until the next replay)."""
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):  # a graph launches on the current stream
            self.graph.replay()
        self.stream.synchronize()
        self._check()
        total = int(self.info[0])
        if self.fmt == "csr" and total > 0x7fffffff:
            raise ValueError(f"{total} pairs do not fit the int32 indptr of SparseCSR")
        if total > self.cap:  # denser than recorded: emit again into larger buffers, record again
            self._alloc_out(self._grown(total))
            with torch.cuda.stream(self.stream):
                self._emit()
            self.stream.synchronize()
            self._record()
        return dict(row=None if self.row is None else self.row[:total], col=self.col[:total], offsets=self.offsets,
                    indptr=self.indptr, counts=self.counts[:self.nq], total=total, info=self.info.clone())


class StaticSearch:
    """``radiusSearch(..., algorithm='compact')`` of one cloud whose size stays fixed, replayed as a
    CUDA graph: ``update()`` copies new positions (and supports) into the plan's buffers, ``run()``
    searches and returns the ``SparseCOO`` / ``SparseCSR`` that ``radiusSearch`` would."""

    def __init__(self, pointCloud: PointCloud, domain: DomainDescription, mode: str = "gather",
                 hashMapLength: int = 4096, format: str = "csr", device=None):
        pos = pointCloud.positions
        dev = _require_cuda(torch.device(device) if device is not None else pos.device)
        self.device = dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.dim = int(pos.shape[1])
        self.n = int(pos.shape[0])
        self.format = format
        self.pos = _as_f32(pos, self.device).clone()
        if pointCloud.supports is None:
            raise ValueError("StaticSearch needs per-point supports")
        self.sup = _as_f32(pointCloud.supports, self.device).clone()
        lo, hi, mask = _domain_host(domain, self.dim)
        t = cloud_table(1)
        t["dim"] = self.dim
        t["periodic_mask"] = mask
        t["domain_min"][0, :self.dim] = lo
        t["domain_max"][0, :self.dim] = hi
        t["hash_map_length"] = int(hashMapLength)
        t["n_query"] = t["n_ref"] = self.n
        t["query_pos"] = t["ref_pos"] = self.pos.data_ptr()
        t["query_sup"] = t["ref_sup"] = self.sup.data_ptr()
        self.plan = SearchPlan(t, mode, True, format, self.device)

    def update(self, positions: torch.Tensor, supports: Optional[torch.Tensor] = None):
        """Copies new positions (and supports) into the plan's input buffers (on its stream, after
        the caller's stream has produced them)."""
        user = torch.cuda.current_stream(self.device)
        self.plan.stream.wait_stream(user)
        with torch.cuda.stream(self.plan.stream):
            for dst, src in ((self.pos, positions), (self.sup, supports)):
                if src is None:
                    continue
                if src.device.type == "cuda":
                    src.record_stream(self.plan.stream)
                dst.copy_(src, non_blocking=True)

    def run(self):
        out = self.plan.replay()
        if self.format == "coo":
            return SparseCOO(out["row"], out["col"], self.n, self.n)
        return SparseCSR(out["col"], out["indptr"], out["counts"], self.n, self.n)
