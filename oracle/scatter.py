"""Test infrastructure: a numpy restatement of the reference's CPU scatter operators.

The checker for ``torchcompactradius_b200.scatter`` (never imported by the product).  It follows
src/torchCompactRadius/cppSrc/sparseOperations:
  * scatter_cpu.cpp:56-77 -- src viewed as [B][E][K]; out starts at Reducer<>::init() unless an
    out tensor is given; the elements are folded in row-major order, so every output element sees
    its elements in increasing e;
  * reducer.h:44-66 -- the folds: sum / mean add, mul multiplies, min / max replace on a strict
    `<` / `>` and record e in arg_out (initialised to E = src.size(dim));
  * scatter_cpu.cpp:74-75 -- without an out tensor, min / max outputs still equal to the type's
    max / lowest become 0;
  * scatter_cpu.cpp:45-49 -- no elements at all: out (when not given) is 0, for every reduce;
  * scatterWrapper.cpp:121-146 -- mean: the sum above, divided by the count of elements per
    output counted in src's dtype (a scatter_sum of ones), below 1 taken as 1; true division for
    floating types, floor division for integers.
Element arithmetic rounds like the reference's CPU types: numpy float16 computes in float32 and
rounds after each operation as c10::Half does; bfloat16 (which numpy lacks) is carried in float32
arrays and rounded to nearest even after each operation, as c10::BFloat16 does; integer arrays
wrap.  Pinned to the reference's own compiled operators by the fixtures in
tests/golden/scatter_cases.npz (tests/test_scatter_oracle.py).
"""
import numpy as np

INT_LIMITS = {np.dtype(t): (np.iinfo(t).max, np.iinfo(t).min) for t in
              (np.uint8, np.int8, np.int16, np.int32, np.int64)}


def round_bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), kept in float32."""
    x = np.asarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), np.float32(np.nan), out).astype(np.float32)


def _limits(dtype, bf16):
    if bf16:
        big = np.uint32(0x7F7F0000).view(np.float32)
        return np.float32(big), np.float32(-big)
    if dtype.kind == "f":
        fi = np.finfo(dtype)
        return dtype.type(fi.max), dtype.type(fi.min)
    hi, lo = INT_LIMITS[dtype]
    return dtype.type(hi), dtype.type(lo)


def scatter(src, index_b, dim, reduce, out=None, dim_size=None, bf16=False):
    """One reduction.  src: numpy array (bfloat16 values as float32 with bf16=True); index_b: int64
    index already broadcast to src's shape; out: optional start values (copied).  Returns
    (out, arg_out or None)."""
    src = np.asarray(src)
    index_b = np.broadcast_to(np.asarray(index_b, dtype=np.int64), src.shape)
    dt = src.dtype
    nd = src.ndim
    dim = dim + nd if dim < 0 else dim
    shape = list(src.shape)
    B = int(np.prod(shape[:dim], dtype=np.int64))
    E = shape[dim]
    K = int(np.prod(shape[dim + 1:], dtype=np.int64))
    if out is not None:
        N = out.shape[dim]
    elif dim_size is not None:
        N = int(dim_size)
    else:
        N = 0 if index_b.size == 0 else int(index_b.max()) + 1
    oshape = list(shape)
    oshape[dim] = N
    hi, lo = _limits(dt, bf16)
    init = {"sum": dt.type(0), "mean": dt.type(0), "mul": dt.type(1), "min": hi, "max": lo}[reduce]
    minmax = reduce in ("min", "max")
    arg = np.full(oshape, E, dtype=np.int64) if minmax else None
    if src.size == 0:
        res = np.array(out, copy=True) if out is not None else np.zeros(oshape, dtype=dt)
        return res, arg
    o3 = (np.array(out, copy=True).reshape(B, N, K) if out is not None else np.full((B, N, K), init, dtype=dt))
    a3 = arg.reshape(B, N, K) if minmax else None
    c3 = np.zeros((B, N, K), dtype=dt)
    s3 = src.reshape(B, E, K)
    i3 = index_b.reshape(B, E, K)
    bb, kk = np.meshgrid(np.arange(B), np.arange(K), indexing="ij")
    rnd = round_bf16 if bf16 else (lambda v: v)
    with np.errstate(all="ignore"):
        for e in range(E):
            v = s3[:, e, :]
            n = i3[:, e, :]
            cur = o3[bb, n, kk]
            if reduce in ("sum", "mean"):
                o3[bb, n, kk] = rnd(cur + v)
                if reduce == "mean":
                    c3[bb, n, kk] = rnd(c3[bb, n, kk] + dt.type(1))
            elif reduce == "mul":
                o3[bb, n, kk] = rnd(cur * v)
            else:
                take = (v < cur) if reduce == "min" else (v > cur)
                o3[bb, n, kk] = np.where(take, v, cur)
                a3[bb, n, kk] = np.where(take, e, a3[bb, n, kk])
        if reduce == "mean":
            c3 = np.where(c3 < dt.type(1), dt.type(1), c3).astype(dt)
            if dt.kind == "f":
                o3 = rnd((o3 / c3).astype(dt))
            else:
                o3 = (o3 // c3).astype(dt)
    if minmax and out is None:
        o3 = np.where(o3 == init, dt.type(0), o3).astype(dt)
    return o3.reshape(oshape), arg
