"""Reductions of values onto an index: the reference's scatter operators on the device.

``scatter_sum``, ``scatter_mul``, ``scatter_mean``, ``scatter_min`` and ``scatter_max`` take the
arguments of the reference's operators (src/torchCompactRadius/cppSrc/sparseOperations/scatter.h:
10-36, registered as torch operators in cppSrc/cppWrapper.cpp:54-58): ``src``, an int64 ``index``
broadcast against ``src`` along ``dim`` (sparseOperations/scatterWrapper.cpp:18-26), ``dim``, an
optional ``out`` that the elements are reduced into, and an optional ``dim_size``.  ``out[.., n,
..]`` reduces every element of ``src`` whose index is ``n``; without ``out`` its size along ``dim``
is ``dim_size`` or ``index.max() + 1``.  ``scatter_min`` / ``scatter_max`` return ``(out,
arg_out)``, ``arg_out`` the position along ``dim`` of the kept element or ``src.size(dim)`` where
none landed, and put 0 where none landed.  Gradients are the reference's
(scatterWrapper.cpp:44-242).

The reduction runs in ``tcr_scatter`` (``csrc/tcr_scatter.cu``): every output element folds its
elements in increasing position in the element type's arithmetic, so the sums, products and means
equal the reference's CPU operators bit for bit (its CUDA operators add with atomics in arrival
order) and repeat from run to run.  Inputs on the CPU are reduced on the current CUDA device and
the result comes back to the CPU; there is no CPU implementation.
"""
import ctypes
import math
from typing import Optional, Tuple

import torch

from . import _lib
from .search import _ptr, _require_cuda

DTYPES = {torch.uint8: 0, torch.int8: 1, torch.int16: 2, torch.int32: 3, torch.int64: 4, torch.float16: 5,
          torch.bfloat16: 6, torch.float32: 7, torch.float64: 8}


def broadcast(index: torch.Tensor, src: torch.Tensor, dim: int) -> torch.Tensor:
    """The reference's index broadcast (scatterWrapper.cpp:18-26): a 1-D index is placed along
    ``dim``, trailing dimensions are added, and the result is expanded to ``src``'s shape."""
    if index.dim() == 1:
        for _ in range(dim):
            index = index.unsqueeze(0)
    for _ in range(index.dim(), src.dim()):
        index = index.unsqueeze(-1)
    return index.expand(src.size())


def index_stats(index: torch.Tensor, stream=None) -> Tuple[int, int, int]:
    """(min, max, descents) of a contiguous int64 CUDA tensor, read back to the host (one sync);
    descents counts the positions whose value is below the previous one."""
    dev = index.device
    stats = torch.empty(3, dtype=torch.int64, device=dev)
    host = torch.empty(3, dtype=torch.int64, pin_memory=True)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    _lib.check(_lib.load().tcr_index_stats(_ptr(index), index.numel(), _ptr(stats), ctypes.c_void_p(host.data_ptr()),
                                           ctypes.c_void_p(st.cuda_stream)), "tcr_index_stats")
    st.synchronize()
    return int(host[0]), int(host[1]), int(host[2])


def _norm_dim(dim: int, nd: int) -> int:
    if nd == 0:
        raise RuntimeError("scatter needs a src with at least one dimension")
    d = dim + nd if dim < 0 else dim
    if d < 0 or d >= nd:
        raise IndexError(f"dim {dim} is out of range for a {nd}-dimensional src")
    return d


def _scatter(src: torch.Tensor, index: torch.Tensor, dim: int, out: Optional[torch.Tensor],
             dim_size: Optional[int], reduce: str):
    """Forward of one reduction; returns (out, arg_out or None, broadcast index, normalised dim)."""
    if not isinstance(index, torch.Tensor) or index.dtype != torch.int64:
        raise RuntimeError("index must be an int64 tensor")
    if src.dtype not in DTYPES:
        raise RuntimeError(f"scatter does not support dtype {src.dtype}")
    dim = _norm_dim(dim, src.dim())
    index_b = broadcast(index, src, dim)  # expand raises for shapes that do not broadcast
    if out is not None:
        if out.dim() != src.dim() or any(out.size(i) != src.size(i) for i in range(src.dim()) if i != dim):
            raise RuntimeError("Input mismatch: out must have src's sizes outside dim")
        if out.dtype != src.dtype:
            raise RuntimeError(f"out has dtype {out.dtype}, src {src.dtype}")
    in_device = src.device
    device = _require_cuda(in_device)
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    shape = list(src.shape)
    B = math.prod(shape[:dim])
    E = shape[dim]
    K = math.prod(shape[dim + 1:])
    src_d = src.detach().to(device).contiguous()
    idx_d = index_b.detach().to(device)
    one_d = all(idx_d.stride(i) == 0 or idx_d.size(i) == 1 for i in range(idx_d.dim()) if i != dim)
    if one_d:  # the index depends on the position along dim only
        sel = tuple(0 if i != dim else slice(None) for i in range(idx_d.dim()))
        idx_d = idx_d[sel].contiguous()
    else:
        idx_d = idx_d.contiguous().reshape(-1)
    nel = B * E * K
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream(device)
        known = out is not None or dim_size is not None
        if out is not None:
            N = out.size(dim)
        elif dim_size is not None:
            N = int(dim_size)
        else:  # the size comes from the index: read its statistics first (the reference's index.max())
            lo, hi, descents = index_stats(idx_d, stream) if idx_d.numel() > 0 else (0, -1, 0)
            N = 0 if index_b.numel() == 0 else hi + 1
        if N < 0:
            raise RuntimeError(f"dim_size {N} is negative")
        if nel > 0 and N == 0:
            raise IndexError("index values must lie in [0, 0): the output is empty")
        shape[dim] = N
        if out is not None:
            out_d = out.detach()
            if out_d.device != device or not out_d.is_contiguous():
                out_d = out_d.to(device).contiguous()
        else:
            out_d = torch.empty(shape, dtype=src.dtype, device=device)
        minmax = reduce in ("min", "max")
        arg_d = torch.empty(shape, dtype=torch.int64, device=device) if minmax else None
        d = _lib.ScatterDesc()
        d.reduce = _lib.REDUCE[reduce]
        d.dtype = DTYPES[src.dtype]
        d.index_full = 0 if one_d else 1
        d.accumulate = 1 if out is not None else 0
        d.B, d.E, d.K, d.N = B, E, K, N
        d.src = src_d.data_ptr() if src_d.numel() else None
        d.index = idx_d.data_ptr() if idx_d.numel() else None
        d.out = out_d.data_ptr() if out_d.numel() else None
        d.arg_out = arg_d.data_ptr() if (arg_d is not None and arg_d.numel()) else None
        lib = _lib.load()
        sp = ctypes.c_void_p(stream.cuda_stream)

        def call(index_sorted, stats_host):
            d.index_sorted = index_sorted
            scratch = torch.empty(max(_lib.scatter_sizes(d), 1), dtype=torch.uint8, device=device)
            _lib.check(lib.tcr_scatter(ctypes.byref(d), _ptr(scratch), scratch.numel(), stats_host, sp),
                       "tcr_scatter")

        if nel == 0:
            call(0, None)
        elif known:
            # One pass when the index is in order (the rows of a neighbour list): the kernels check
            # it while reading it and write nothing when it descends or leaves [0, N).
            host = torch.empty(3, dtype=torch.int64, pin_memory=True)
            call(1 if one_d else 0, ctypes.c_void_p(host.data_ptr()))
            stream.synchronize()
            lo, hi, descents = int(host[0]), int(host[1]), int(host[2])
            if lo < 0 or hi >= N:
                raise IndexError(f"index values must lie in [0, {N}) (found {lo} .. {hi})")
            if one_d and descents > 0:
                call(0, None)
        else:
            if lo < 0:
                raise IndexError(f"index values must lie in [0, {N}) (found {lo} .. {hi})")
            call(1 if (one_d and descents == 0) else 0, None)
    if out is not None:
        if out_d.data_ptr() != out.data_ptr():
            out.copy_(out_d)
        res = out
    else:
        res = out_d if in_device.type == "cuda" else out_d.to(in_device)
    arg = None
    if arg_d is not None:
        arg = arg_d if in_device.type == "cuda" else arg_d.to(in_device)
    return res, arg, index_b, dim


class _ScatterSum(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, index, dim, out, dim_size):
        res, _, index_b, d = _scatter(src, index, dim, out, dim_size, "sum")
        ctx.save_for_backward(index_b)
        ctx.dim = d
        if out is not None:
            ctx.mark_dirty(out)
        return res

    @staticmethod
    def backward(ctx, grad_out):  # scatterWrapper.cpp:60-68
        (index_b,) = ctx.saved_tensors
        return torch.gather(grad_out, ctx.dim, index_b), None, None, None, None


class _ScatterMul(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, index, dim, out, dim_size):
        res, _, index_b, d = _scatter(src, index, dim, out, dim_size, "mul")
        ctx.save_for_backward(src, index_b, res)
        ctx.dim = d
        if out is not None:
            ctx.mark_dirty(out)
        return res

    @staticmethod
    def backward(ctx, grad_out):  # scatterWrapper.cpp:92-103
        src, index_b, res = ctx.saved_tensors
        grad_in = torch.gather(grad_out * res, ctx.dim, index_b).div_(src)
        grad_in.masked_fill_(grad_in.isnan(), 0)
        return grad_in, None, None, None, None


class _ScatterMean(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, index, dim, out, dim_size):
        res, _, index_b, d = _scatter(src, index, dim, out, dim_size, "mean")
        ctx.save_for_backward(index_b)
        ctx.dim = d
        ctx.n = res.size(d)
        if out is not None:
            ctx.mark_dirty(out)
        return res

    @staticmethod
    def backward(ctx, grad_out):  # scatterWrapper.cpp:121-160: count of elements per output, at least 1
        (index_b,) = ctx.saved_tensors
        ones = torch.ones(index_b.shape, dtype=grad_out.dtype, device=grad_out.device)
        count = _scatter(ones, index_b, ctx.dim, None, ctx.n, "sum")[0]
        count.masked_fill_(count < 1, 1)
        grad_in = torch.gather(grad_out, ctx.dim, index_b)
        grad_in.true_divide_(torch.gather(count, ctx.dim, index_b))
        return grad_in, None, None, None, None


class _ScatterMinMax(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, index, dim, out, dim_size, reduce):
        res, arg, index_b, d = _scatter(src, index, dim, out, dim_size, reduce)
        ctx.save_for_backward(index_b, arg)
        ctx.dim = d
        ctx.src_shape = list(src.shape)
        ctx.mark_non_differentiable(arg)
        if out is not None:
            ctx.mark_dirty(out)
        return res, arg

    @staticmethod
    def backward(ctx, grad_out, grad_arg):  # scatterWrapper.cpp:178-190, 211-223
        _, arg = ctx.saved_tensors
        shape = list(ctx.src_shape)
        shape[ctx.dim] += 1
        grad_in = torch.zeros(shape, dtype=grad_out.dtype, device=grad_out.device)
        grad_in.scatter_(ctx.dim, arg, grad_out)
        grad_in = grad_in.narrow(ctx.dim, 0, shape[ctx.dim] - 1)
        return grad_in, None, None, None, None, None


def scatter_sum(src: torch.Tensor, index: torch.Tensor, dim: int = -1, out: Optional[torch.Tensor] = None,
                dim_size: Optional[int] = None) -> torch.Tensor:
    """Sum of the elements landing on every output position (reference scatter_sum)."""
    return _ScatterSum.apply(src, index, dim, out, dim_size)


def scatter_mul(src: torch.Tensor, index: torch.Tensor, dim: int = -1, out: Optional[torch.Tensor] = None,
                dim_size: Optional[int] = None) -> torch.Tensor:
    """Product of the elements landing on every output position, 1 where none land."""
    return _ScatterMul.apply(src, index, dim, out, dim_size)


def scatter_mean(src: torch.Tensor, index: torch.Tensor, dim: int = -1, out: Optional[torch.Tensor] = None,
                 dim_size: Optional[int] = None) -> torch.Tensor:
    """Sum divided by the count of landing elements (at least 1), in src's dtype (floor division
    for integers), as the reference's scatter_mean."""
    return _ScatterMean.apply(src, index, dim, out, dim_size)


def scatter_min(src: torch.Tensor, index: torch.Tensor, dim: int = -1, out: Optional[torch.Tensor] = None,
                dim_size: Optional[int] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """(smallest landing element, its position along dim); the first of equal values is kept."""
    return _ScatterMinMax.apply(src, index, dim, out, dim_size, "min")


def scatter_max(src: torch.Tensor, index: torch.Tensor, dim: int = -1, out: Optional[torch.Tensor] = None,
                dim_size: Optional[int] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """(largest landing element, its position along dim); the first of equal values is kept."""
    return _ScatterMinMax.apply(src, index, dim, out, dim_size, "max")
