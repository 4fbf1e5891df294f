"""`vector::*` algorithms of massively over the C ABI.

Each function mirrors the public function of massively/src/api/algorithm/
named in its docstring (same argument order and meaning, same errors) and
runs on the executor's stream through libmassively_b200.so.  Inputs may be
DeviceVecs, lazy views (massively_b200.lazy) or zips of them; outputs are
new DeviceVecs (zips for multi-column rows).  Length-changing results carry
their count on the device (DeviceVec.len_dev), as massively's
LogicalExtent::Device does, so pipelines need no host synchronisation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from . import op as O
from .iter import Zip
from .lazy import Map, View, lower
from .runtime import (ID_TO_NP, DeviceVec, Executor, ForeignExecutor, LengthMismatch,
                      LengthTooLarge, MINDEX_MAX, check, scalar_buffer)

_L = N.lib


def _columns(x) -> list:
    return list(x.cols) if isinstance(x, Zip) else [x]


def _srcs(exec: Executor, x, keep: list):
    cols = _columns(x)
    arr = (N.mb_src * len(cols))()
    for k, c in enumerate(cols):
        arr[k] = lower(exec, c, keep)
    return arr, len(cols)


def _out_like(exec: Executor, x, n: int, len_dev=None):
    outs = []
    for c in _columns(x):
        v = exec.alloc(c.dtype, n)
        if len_dev is not None:
            v = v.with_len_dev(len_dev)
        outs.append(v)
    return outs


def _cols(outs) -> C.Array:
    arr = (N.mb_col * len(outs))()
    for k, o in enumerate(outs):
        arr[k] = o.to_col()
    return arr


def _wrap(x, outs):
    return Zip(*outs) if isinstance(x, Zip) else outs[0]


def _check_owner(exec: Executor, *xs):
    for x in xs:
        for c in _columns(x):
            if isinstance(c, DeviceVec) and c.owner != exec.id:
                raise ForeignExecutor()


def _len(x) -> int:
    n = len(x)
    if n > MINDEX_MAX:
        raise LengthTooLarge(n)
    return n


def _dtype(x):
    return _columns(x)[0].dtype


def _len_dev_of(x):
    c = _columns(x)[0]
    return c.len_dev if isinstance(c, DeviceVec) else None


def _first_len_dev(*xs):
    # (never truth-test a device tensor: that reads it back, a sync)
    for x in xs:
        ld = _len_dev_of(x)
        if ld is not None:
            return ld
    return None


def _count_buffer(exec: Executor) -> torch.Tensor:
    t = exec.storage(torch.uint32, 1)
    t.zero_()
    return t


def _p32(t: torch.Tensor):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_uint32))


# ------------------------------------------------------------ transform --

def copy(exec: Executor, input, output: DeviceVec) -> None:
    """vector::copy (massively/src/api/algorithm/transform.rs:56)."""
    keep = []
    s = lower(exec, input, keep)
    check(_L().mb_copy(exec.handle, C.byref(s), output.to_col()))


def _plain(exec: Executor, input, dtype) -> DeviceVec:
    """The input as a plain column of `dtype` (lazy views are materialised)."""
    if isinstance(input, DeviceVec) and input.dtype == dtype and input.len_dev is None:
        return input
    from .lazy import Map as _Map
    out = exec.alloc(dtype, _len(input))
    copy(exec, _Map(input, O.Identity, dtype), out)
    return out


def map(exec: Executor, input, unary, dtype=None) -> DeviceVec:  # noqa: A001
    """vector::map (transform.rs:91-110) for a built-in unary op or a
    compiled user map (op.UserOp.map)."""
    if isinstance(unary, O.UserOp):
        _check_owner(exec, input)
        x = _plain(exec, input, unary.dtype)
        out = exec.alloc(unary.out_dtype, len(x))
        check(_L().mb_map_user(exec.handle, C.byref(x.to_src()), unary.handle, out.to_col()))
        return out
    from .lazy import Map
    v = Map(input, unary, dtype)
    out = exec.alloc(v.dtype, len(v))
    copy(exec, v, out)
    return out


def fill(exec: Executor, value, output: DeviceVec) -> None:
    """vector::fill (selection.rs:321)."""
    buf = scalar_buffer(value, output.dtype)
    check(_L().mb_fill(exec.handle, buf, output.to_col()))


def replace_where(exec: Executor, value, stencil, output) -> None:
    """vector::replace_where (massively/src/api/algorithm/selection.rs:363):
    output items whose stencil flag is non-zero become `value` (a tuple for
    zipped outputs); the others keep theirs."""
    _check_owner(exec, stencil, output)
    from .runtime import value_bits
    cols = _columns(output)
    vals = list(value) if isinstance(value, (tuple, list)) else [value]
    if len(vals) != len(cols):
        raise LengthMismatch(len(cols), len(vals))
    keep = []
    st = lower(exec, stencil, keep)
    bits = (C.c_uint64 * len(cols))(*[value_bits(v, c.dtype) for v, c in zip(vals, cols)])
    check(_L().mb_replace_where(exec.handle, bits, C.byref(st), _cols(cols), len(cols)))


def transform_where(exec: Executor, input, unary, stencil, output) -> None:
    """vector::transform_where (selection.rs:436): output[i] = unary(input[i])
    where the stencil flag is non-zero; other items keep theirs.  `unary` a
    built-in op (op.UnaryOp) applied to every column of a zipped input."""
    _check_owner(exec, input, stencil, output)
    ins, outs = _columns(input), _columns(output)
    if len(ins) != len(outs):
        raise LengthMismatch(len(ins), len(outs))
    keep = []
    views = [Map(c, unary, o.dtype) for c, o in zip(ins, outs)]
    srcs = (N.mb_src * len(views))(*[lower(exec, v, keep) for v in views])
    st = lower(exec, stencil, keep)
    check(_L().mb_transform_where(exec.handle, srcs, len(views), C.byref(st), _cols(outs)))


# ----------------------------------------------------------------- scan --

def inclusive_scan(exec: Executor, input, op) -> DeviceVec:
    """vector::inclusive_scan (massively/src/api/algorithm/scan.rs:96); `op`
    a built-in or a compiled user operator (op.UserOp.binary)."""
    _check_owner(exec, input)
    if isinstance(op, O.UserOp):
        x = _plain(exec, input, op.dtype)
        out = exec.alloc(op.dtype, len(x))
        check(_L().mb_inclusive_scan_user(exec.handle, C.byref(x.to_src()), op.handle,
                                          out.to_col()))
        return out
    keep = []
    n = _len(input)
    s = lower(exec, input, keep)
    out = exec.alloc(_dtype(input), n)
    if s.len_dev:
        out = out.with_len_dev(_len_dev_of(input))
    check(_L().mb_inclusive_scan(exec.handle, C.byref(s), O.reduction(op).id, out.to_col()))
    return out


def exclusive_scan(exec: Executor, input, init, op) -> DeviceVec:
    """vector::exclusive_scan (scan.rs:216)."""
    _check_owner(exec, input)
    if isinstance(op, O.UserOp):
        x = _plain(exec, input, op.dtype)
        out = exec.alloc(op.dtype, len(x))
        buf = scalar_buffer(init, op.dtype)
        check(_L().mb_exclusive_scan_user(exec.handle, C.byref(x.to_src()), op.handle, buf,
                                          out.to_col()))
        return out
    keep = []
    n = _len(input)
    s = lower(exec, input, keep)
    out = exec.alloc(_dtype(input), n)
    if s.len_dev:
        out = out.with_len_dev(_len_dev_of(input))
    buf = scalar_buffer(init, _dtype(input))
    check(_L().mb_exclusive_scan(exec.handle, C.byref(s), O.reduction(op).id, buf,
                                 out.to_col()))
    return out


def inclusive_scan_into(exec: Executor, input, op, output: DeviceVec) -> None:
    """inclusive_scan into caller storage (scan.rs:117)."""
    keep = []
    s = lower(exec, input, keep)
    check(_L().mb_inclusive_scan(exec.handle, C.byref(s), O.reduction(op).id, output.to_col()))


def exclusive_scan_into(exec: Executor, input, init, op, output: DeviceVec) -> None:
    keep = []
    s = lower(exec, input, keep)
    buf = scalar_buffer(init, _dtype(input))
    check(_L().mb_exclusive_scan(exec.handle, C.byref(s), O.reduction(op).id, buf,
                                 output.to_col()))


def adjacent_difference(exec: Executor, input, op) -> DeviceVec:
    """vector::adjacent_difference (scan.rs:156)."""
    from .lazy import AdjacentDifference, _as_column
    keep = []
    return _as_column(exec, AdjacentDifference(input, op), keep)


# --------------------------------------------------------------- reduce --

def reduce(exec: Executor, input, init, op):
    """vector::reduce (massively/src/api/algorithm/reduce.rs:32-50): returns
    `init op fold(input)` on the host (synchronises); `op` a built-in or a
    compiled user operator (op.UserOp.binary)."""
    _check_owner(exec, input)
    if isinstance(op, O.UserOp):
        x = _plain(exec, input, op.dtype)
        buf = scalar_buffer(init, op.dtype)
        res = np.zeros(1, dtype=op.dtype)
        check(_L().mb_reduce_user(exec.handle, C.byref(x.to_src()), op.handle, buf, None,
                                  res.ctypes.data_as(C.c_void_p)))
        return res[0]
    keep = []
    _len(input)
    s = lower(exec, input, keep)
    dt = ID_TO_NP[s.vtype]
    buf = scalar_buffer(init, dt)
    res = np.zeros(1, dtype=dt)
    check(_L().mb_reduce(exec.handle, C.byref(s), O.reduction(op).id, buf, None,
                         res.ctypes.data_as(C.c_void_p)))
    return res[0]


def reduce_to_device(exec: Executor, input, init, op) -> DeviceVec:
    """reduce whose single result stays on the device (no synchronisation)."""
    keep = []
    s = lower(exec, input, keep)
    dt = ID_TO_NP[s.vtype]
    out = exec.alloc(dt, 1)
    buf = scalar_buffer(init, dt)
    check(_L().mb_reduce(exec.handle, C.byref(s), O.reduction(op).id, buf,
                         C.c_void_p(out.data_ptr()), None))
    return out


# ------------------------------------------------------------ selection --

def _stencil_src(exec, stencil, keep):
    return lower(exec, stencil, keep)


def copy_where(exec: Executor, input, stencil):
    """vector::copy_where (massively/src/api/algorithm/selection.rs:146):
    rows whose stencil flag is non-zero, stable; the count stays on device."""
    return _select(exec, input, stencil, remove=False)


def remove_where(exec: Executor, input, stencil):
    """vector::remove_where (selection.rs:203)."""
    return _select(exec, input, stencil, remove=True)


def _select(exec, input, stencil, remove):
    _check_owner(exec, input, stencil)
    n, m = _len(input), _len(stencil)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    srcs, k = _srcs(exec, input, keep)
    st = _stencil_src(exec, stencil, keep)
    cnt = _count_buffer(exec)
    outs = _out_like(exec, input, n, cnt)
    fn = _L().mb_remove_where if remove else _L().mb_copy_where
    check(fn(exec.handle, srcs, k, C.byref(st), _cols(outs), _p32(cnt), None))
    return _wrap(input, outs)


def partition(exec: Executor, input, pred, column: int = 0):
    """vector::partition (selection.rs:272): (rows where pred holds, then the
    rest, both stable; boundary).  `column` picks the zipped column tested."""
    _check_owner(exec, input)
    n = _len(input)
    keep = []
    srcs, k = _srcs(exec, input, keep)
    outs = _out_like(exec, input, n)
    b = C.c_uint32(0)
    check(_L().mb_partition(exec.handle, srcs, k, column, O.unary(pred).id, _cols(outs), None,
                            C.byref(b)))
    return _wrap(input, outs), int(b.value)


# ------------------------------------------------------- gather/scatter --

def gather(exec: Executor, values, indices):
    """vector::gather (massively/src/api/algorithm/indexed.rs:172)."""
    _check_owner(exec, values, indices)
    n = _len(indices)
    outs = _out_like(exec, values, n)
    _gather_into(exec, values, indices, None, outs)
    return _wrap(values, outs)


def gather_where(exec: Executor, values, indices, stencil, output) -> None:
    """vector::gather_where (indexed.rs:237): writes only where stencil != 0."""
    _check_owner(exec, values, indices, stencil, output)
    n, m = _len(indices), _len(stencil)
    if n != m:
        raise LengthMismatch(n, m)
    _gather_into(exec, values, indices, stencil, _columns(output))


def _gather_into(exec, values, indices, stencil, outs):
    keep = []
    idx = lower(exec, indices, keep)
    st = lower(exec, stencil, keep) if stencil is not None else None
    for c, o in zip(_columns(values), outs):
        s = lower(exec, c, keep)
        check(_L().mb_gather(exec.handle, C.byref(s), C.byref(idx),
                             C.byref(st) if st is not None else None, o.to_col()))


def scatter(exec: Executor, values, indices, output) -> None:
    """vector::scatter (massively/src/api/algorithm/scatter.rs:248)."""
    _check_owner(exec, values, indices, output)
    n, m = _len(values), _len(indices)
    if n != m:
        raise LengthMismatch(n, m)
    _scatter_into(exec, values, indices, None, _columns(output))


def scatter_where(exec: Executor, values, indices, stencil, output) -> None:
    """vector::scatter_where (scatter.rs:315)."""
    _check_owner(exec, values, indices, stencil, output)
    n, m = _len(values), _len(indices)
    if n != m:
        raise LengthMismatch(n, m)
    _scatter_into(exec, values, indices, stencil, _columns(output))


def _scatter_into(exec, values, indices, stencil, outs):
    keep = []
    idx = lower(exec, indices, keep)
    st = lower(exec, stencil, keep) if stencil is not None else None
    for c, o in zip(_columns(values), outs):
        s = lower(exec, c, keep)
        check(_L().mb_scatter(exec.handle, C.byref(s), C.byref(idx),
                              C.byref(st) if st is not None else None, o.to_col()))


def scatter_reduce(exec: Executor, values, indices, init, op, output) -> None:
    """vector::scatter_reduce (massively/src/api/algorithm/scatter.rs:377):
    out[d] = out[d] op (init op v ...) for every destination named by
    `indices`; other destinations keep their value.  `op` must be associative
    and commutative; for zipped values / outputs `op` and `init` may be
    per-column tuples."""
    _check_owner(exec, values, indices, output)
    n, m = _len(values), _len(indices)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    vs, nv = _srcs(exec, values, keep)
    ix = lower(exec, indices, keep)
    outs = _columns(output)
    if len(outs) != nv:
        raise LengthMismatch(nv, len(outs))
    ids, bits = _ops_inits(values, op, init)
    check(_L().mb_scatter_reduce(exec.handle, vs, nv, C.byref(ix), ids, bits, _cols(outs)))


def reverse(exec: Executor, values):
    """vector::reverse (indexed.rs:289)."""
    from .lazy import Reverse
    outs = []
    for c in _columns(values):
        o = exec.alloc(c.dtype, len(c))
        copy(exec, Reverse(c, len(c)), o)
        outs.append(o)
    return _wrap(values, outs)


# ------------------------------------------------------------- ordering --

def radix_sort_by_key(exec: Executor, keys, values):
    """vector::radix_sort_by_key (massively/src/api/algorithm/by_key.rs:272):
    the values permuted into the stable radix order of the keys (1-3 key
    columns, the first primary)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks, nk = _srcs(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    outs = _out_like(exec, values, n, _first_len_dev(keys, values))
    check(_L().mb_radix_sort_by_key(exec.handle, ks, nk, vs, nv, _cols(outs), None))
    return _wrap(values, outs)


def radix_sort_pairs(exec: Executor, keys, values):
    """Sorted keys and values together (one onesweep pass set)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks, nk = _srcs(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    ld = _first_len_dev(keys, values)  # a device count carries over
    kout = _out_like(exec, keys, n, ld)
    vout = _out_like(exec, values, n, ld)
    check(_L().mb_radix_sort_by_key(exec.handle, ks, nk, vs, nv, _cols(vout), _cols(kout)))
    return _wrap(keys, kout), _wrap(values, vout)


def sort(exec: Executor, input, less=O.Less) -> DeviceVec:
    """vector::sort (massively/src/api/algorithm/ordering.rs:64): stable;
    `less` a built-in predicate or a compiled comparator
    (op.UserOp.predicate)."""
    _check_owner(exec, input)
    if isinstance(less, O.UserOp):
        x = _plain(exec, input, less.dtype)
        out = exec.alloc(less.dtype, len(x))
        check(_L().mb_sort_user(exec.handle, C.byref(x.to_src()), less.handle, None, 0,
                                out.to_col(), None))
        return out
    keep = []
    _len(input)
    s = lower(exec, input, keep)
    out = exec.alloc(_dtype(input), len(input))
    check(_L().mb_sort(exec.handle, C.byref(s), O.pred2(less).id, out.to_col()))
    return out


def sort_by_key(exec: Executor, keys, values, less=O.Less):
    """vector::sort_by_key (by_key.rs:226): the values in the stable order of
    the keys under `less` (a built-in predicate or a compiled comparator)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    if isinstance(less, O.UserOp):
        x = _plain(exec, keys, less.dtype)
        keep = []
        vs, nv = _srcs(exec, values, keep)
        outs = _out_like(exec, values, n)
        none = N.mb_col()
        check(_L().mb_sort_user(exec.handle, C.byref(x.to_src()), less.handle, vs, nv, none,
                                _cols(outs)))
        return _wrap(values, outs)
    keep = []
    ks = lower(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    outs = _out_like(exec, values, n)
    check(_L().mb_sort_by_key(exec.handle, C.byref(ks), O.pred2(less).id, vs, nv, None,
                              _cols(outs)))
    return _wrap(values, outs)


# --------------------------------------------------------------- by key --

def _ops_inits(values, op, init):
    cols = _columns(values)
    ops = list(op) if isinstance(op, (tuple, list)) else [op] * len(cols)
    inits = list(init) if isinstance(init, (tuple, list)) else [init] * len(cols)
    if len(ops) != len(cols) or len(inits) != len(cols):
        raise LengthMismatch(len(cols), len(ops))
    from .runtime import value_bits
    ids = (C.c_int * len(cols))(*[O.reduction(o).id for o in ops])
    bits = (C.c_uint64 * len(cols))(*[value_bits(i, c.dtype) for i, c in zip(inits, cols)])
    return ids, bits


def reduce_by_key(exec: Executor, keys, values, equal, init, op):
    """vector::reduce_by_key (massively/src/api/algorithm/by_key.rs:618):
    (run keys, per-run init op v...) with the run count on the device.  For
    zipped values `op` / `init` may be per-column tuples."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks = lower(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    ids, bits = _ops_inits(values, op, init)
    cnt = _count_buffer(exec)
    kout = exec.alloc(_dtype(keys), n).with_len_dev(cnt)
    vout = _out_like(exec, values, n, cnt)
    check(_L().mb_reduce_by_key(exec.handle, C.byref(ks), O.pred2(equal).id, vs, nv, ids, bits,
                                kout.to_col(), _cols(vout), _p32(cnt), None))
    return kout, _wrap(values, vout)


def reduce_by_key_segmented(exec: Executor, keys, values, equal, init, op, offsets: DeviceVec):
    """reduce_by_key whose runs also break at the segment starts given by
    `offsets` (segment_count + 1 entries): many independent requests' rows
    reduce in one launch (no massively counterpart; the batched loop uses it)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks = lower(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    ids, bits = _ops_inits(values, op, init)
    cnt = _count_buffer(exec)
    kout = exec.alloc(_dtype(keys), n).with_len_dev(cnt)
    vout = _out_like(exec, values, n, cnt)
    check(_L().mb_reduce_by_key_segmented(
        exec.handle, C.byref(ks), O.pred2(equal).id, vs, nv, ids, bits,
        C.c_void_p(offsets.data_ptr()), len(offsets) - 1, kout.to_col(), _cols(vout), _p32(cnt),
        None))
    return kout, _wrap(values, vout)


def inclusive_scan_by_key(exec: Executor, keys, values, equal, op):
    """vector::inclusive_scan_by_key (by_key.rs:399)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks = lower(exec, keys, keep)
    outs = []
    for c in _columns(values):
        s = lower(exec, c, keep)
        o = exec.alloc(c.dtype, n)
        check(_L().mb_inclusive_scan_by_key(exec.handle, C.byref(ks), O.pred2(equal).id,
                                            C.byref(s), O.reduction(op).id, o.to_col()))
        outs.append(o)
    return _wrap(values, outs)


def exclusive_scan_by_key(exec: Executor, keys, values, equal, init, op):
    """vector::exclusive_scan_by_key (by_key.rs:497)."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks = lower(exec, keys, keep)
    cols = _columns(values)
    inits = list(init) if isinstance(init, (tuple, list)) else [init] * len(cols)
    outs = []
    for c, i in zip(cols, inits):
        s = lower(exec, c, keep)
        o = exec.alloc(c.dtype, n)
        buf = scalar_buffer(i, c.dtype)
        check(_L().mb_exclusive_scan_by_key(exec.handle, C.byref(ks), O.pred2(equal).id,
                                            C.byref(s), O.reduction(op).id, buf, o.to_col()))
        outs.append(o)
    return _wrap(values, outs)


# ---------------------------------------------------------- merge / set --

def unique(exec: Executor, input, equal=O.Equal) -> DeviceVec:
    """vector::unique (massively/src/api/algorithm/ordering.rs:146): the
    first item of every run of equal items; the count stays on the device."""
    _check_owner(exec, input)
    n = _len(input)
    keep = []
    s = lower(exec, input, keep)
    cnt = _count_buffer(exec)
    out = exec.alloc(_dtype(input), n).with_len_dev(cnt)
    check(_L().mb_unique(exec.handle, C.byref(s), O.pred2(equal).id, out.to_col(), _p32(cnt),
                         None))
    return out


def unique_by_key(exec: Executor, keys, values, equal=O.Equal):
    """vector::unique_by_key (by_key.rs:759): the values of the first row of
    every run of equal keys."""
    _check_owner(exec, keys, values)
    n, m = _len(keys), _len(values)
    if n != m:
        raise LengthMismatch(n, m)
    keep = []
    ks = lower(exec, keys, keep)
    vs, nv = _srcs(exec, values, keep)
    cnt = _count_buffer(exec)
    outs = _out_like(exec, values, n, cnt)
    check(_L().mb_unique_by_key(exec.handle, C.byref(ks), vs, nv, O.pred2(equal).id,
                                _cols(outs), _p32(cnt), None))
    return _wrap(values, outs)


def _bounds(exec, source, values, less, fn):
    _check_owner(exec, source, values)
    keep = []
    ss, vs = lower(exec, source, keep), lower(exec, values, keep)
    _len(source)
    out = exec.alloc(np.uint32, _len(values))
    ld = _len_dev_of(values)
    if ld is not None:
        out = out.with_len_dev(ld)
    check(fn(exec.handle, C.byref(ss), C.byref(vs), O.pred2(less).id, out.to_col()))
    return out


def lower_bound(exec: Executor, source, values, less=O.Less) -> DeviceVec:
    """vector::lower_bound (massively/src/api/algorithm/search.rs:81): per
    value, the first index of the sorted source not less than it."""
    return _bounds(exec, source, values, less, _L().mb_lower_bound)


def upper_bound(exec: Executor, source, values, less=O.Less) -> DeviceVec:
    """vector::upper_bound (search.rs:128): per value, the first index of
    the sorted source greater than it."""
    return _bounds(exec, source, values, less, _L().mb_upper_bound)


# ------------------------------------------- predicates and first index --
#
# Each query's result is one u32 on the device: an index (MINDEX_MAX for
# massively's None) or a 0 / 1 flag.  By default it is read back (as
# massively does: "this operation synchronizes to resolve the optional index
# on the host"); with `out` (a u32 DeviceVec, two items for minmax_element)
# it stays on the device, stream-ordered, so the call needs no host
# synchronisation and may sit inside a graph capture.

def _query(exec, fn, inputs, op, out, count=1):
    _check_owner(exec, *inputs)
    keep = []
    srcs = []
    for x in inputs:
        _len(x)
        srcs.append(C.byref(lower(exec, x, keep)))
    if out is not None:
        if out.dtype != np.uint32 or len(out) < count:
            raise ValueError(f"out must be a u32 DeviceVec of at least {count} item(s)")
        check(fn(exec.handle, *srcs, op, _p32(out.tensor), None))
        return None
    res = (C.c_uint32 * 2)()
    check(fn(exec.handle, *srcs, op, None, res))
    return list(res)[:count]


def _opt(r):
    return None if r is None or r == MINDEX_MAX else int(r)


def count(exec: Executor, input) -> int:
    """vector::count (massively/src/api/algorithm/predicate.rs:53): the
    logical number of items -- a device length when the input carries one
    (read back), else its length.  For zipped columns it is the smallest
    logical length of the columns (the rows all of them hold)."""
    _check_owner(exec, input)
    n = _len(input)
    for c in _columns(input):
        if isinstance(c, DeviceVec):
            n = min(n, c.logical_len())
    return n


def count_if(exec: Executor, input, pred) -> int:
    """vector::count_if (massively/src/api/algorithm/predicate.rs:63-90): the
    number of items the predicate passes -- a sum reduction of the
    predicate's 0 / 1 flags (core/predicate.rs:195-202)."""
    _check_owner(exec, input)
    _len(input)
    return int(reduce(exec, Map(input, O.unary(pred)), 0, O.Add))


def all_of(exec: Executor, input, pred) -> bool:
    """vector::all_of (predicate.rs:93-122): count_if == length."""
    return count_if(exec, input, pred) == _len(input)


def any_of(exec: Executor, input, pred) -> bool:
    """vector::any_of (predicate.rs:125-154); answered by the first-index
    search, which stops at the first passing item."""
    return find_if(exec, input, pred) is not None


def none_of(exec: Executor, input, pred) -> bool:
    """vector::none_of (predicate.rs:157-186)."""
    return find_if(exec, input, pred) is None


def find_if(exec: Executor, input, pred, out: DeviceVec | None = None):
    """vector::find_if (predicate.rs:218): the first passing position, or
    None."""
    r = _query(exec, _L().mb_find_if, [input], O.unary(pred).id, out)
    return None if r is None else _opt(r[0])


def is_partitioned(exec: Executor, input, pred, out: DeviceVec | None = None):
    """vector::is_partitioned (predicate.rs:232-260): no passing item after
    a failing one."""
    r = _query(exec, _L().mb_is_partitioned, [input], O.unary(pred).id, out)
    return None if r is None else bool(r[0])


def adjacent_find(exec: Executor, input, equal=O.Equal, out: DeviceVec | None = None):
    """vector::adjacent_find (massively/src/api/algorithm/ordering.rs:107):
    the first i with equal(x[i], x[i+1]), or None."""
    r = _query(exec, _L().mb_adjacent_find, [input], O.pred2(equal).id, out)
    return None if r is None else _opt(r[0])


def is_sorted_until(exec: Executor, input, less=O.Less, out: DeviceVec | None = None):
    """vector::is_sorted_until (ordering.rs:213): the first i with
    less(x[i], x[i-1]), else the length."""
    r = _query(exec, _L().mb_is_sorted_until, [input], O.pred2(less).id, out)
    return None if r is None else int(r[0])


def is_sorted(exec: Executor, input, less=O.Less) -> bool:
    """vector::is_sorted (ordering.rs:256)."""
    return is_sorted_until(exec, input, less) == _len(input)


def find_first_of(exec: Executor, source, needles, equal=O.Equal,
                  out: DeviceVec | None = None):
    """vector::find_first_of (massively/src/api/algorithm/search.rs:33): the
    first source item equal to any needle, or None."""
    r = _query(exec, _L().mb_find_first_of, [source, needles], O.pred2(equal).id, out)
    return None if r is None else _opt(r[0])


def equal(exec: Executor, left, right, eq=O.Equal, out: DeviceVec | None = None):
    """vector::equal (search.rs:175): equal lengths and every pair equal."""
    r = _query(exec, _L().mb_equal, [left, right], O.pred2(eq).id, out)
    return None if r is None else bool(r[0])


def mismatch(exec: Executor, left, right, eq=O.Equal, out: DeviceVec | None = None):
    """vector::mismatch (search.rs:231): the first differing position; past
    an equal common prefix, the shorter length if the lengths differ, else
    None."""
    r = _query(exec, _L().mb_mismatch, [left, right], O.pred2(eq).id, out)
    return None if r is None else _opt(r[0])


def lexicographical_compare(exec: Executor, left, right, less=O.Less,
                            out: DeviceVec | None = None):
    """vector::lexicographical_compare (search.rs:289): left orders before
    right."""
    r = _query(exec, _L().mb_lexicographical_compare, [left, right], O.pred2(less).id, out)
    return None if r is None else bool(r[0])


def min_element(exec: Executor, input, less=O.Less, out: DeviceVec | None = None):
    """vector::min_element (ordering.rs:300-327): the first minimum's index,
    or None."""
    r = _query(exec, _L().mb_min_element, [input], O.pred2(less).id, out)
    return None if r is None else _opt(r[0])


def max_element(exec: Executor, input, less=O.Less, out: DeviceVec | None = None):
    """vector::max_element (ordering.rs:328-360): the first maximum's index,
    or None."""
    r = _query(exec, _L().mb_max_element, [input], O.pred2(less).id, out)
    return None if r is None else _opt(r[0])


def minmax_element(exec: Executor, input, less=O.Less, out: DeviceVec | None = None):
    """vector::minmax_element (ordering.rs:361-412): (last minimum, first
    maximum) as massively's sequential definition keeps them, or None."""
    r = _query(exec, _L().mb_minmax_element, [input], O.pred2(less).id, out, count=2)
    if r is None:
        return None
    return None if r[0] == MINDEX_MAX else (int(r[0]), int(r[1]))


def merge(exec: Executor, left, right, less=O.Less) -> DeviceVec:
    """vector::merge (massively/src/api/algorithm/merge.rs:109)."""
    _check_owner(exec, left, right)
    keep = []
    ls, rs = lower(exec, left, keep), lower(exec, right, keep)
    _len(left), _len(right)
    out = exec.alloc(_dtype(left), len(left) + len(right))
    check(_L().mb_merge(exec.handle, C.byref(ls), C.byref(rs), O.pred2(less).id, out.to_col()))
    return out


def merge_by_key(exec: Executor, left_keys, left_values, right_keys, right_values,
                 less=O.Less):
    """vector::merge_by_key (merge.rs:195): the merged values."""
    _check_owner(exec, left_keys, left_values, right_keys, right_values)
    if len(left_keys) != len(left_values):
        raise LengthMismatch(len(left_keys), len(left_values))
    if len(right_keys) != len(right_values):
        raise LengthMismatch(len(right_keys), len(right_values))
    keep = []
    lk, rk = lower(exec, left_keys, keep), lower(exec, right_keys, keep)
    lv, nv = _srcs(exec, left_values, keep)
    rv, _ = _srcs(exec, right_values, keep)
    n = len(left_keys) + len(right_keys)
    kout = exec.alloc(_dtype(left_keys), n)
    vout = _out_like(exec, left_values, n)
    check(_L().mb_merge_by_key(exec.handle, C.byref(lk), lv, C.byref(rk), rv, nv,
                               O.pred2(less).id, kout.to_col(), _cols(vout)))
    return _wrap(left_values, vout)


def _set(exec, left, right, less, fn, cap):
    _check_owner(exec, left, right)
    keep = []
    ls, rs = lower(exec, left, keep), lower(exec, right, keep)
    cnt = _count_buffer(exec)
    out = exec.alloc(_dtype(left), cap).with_len_dev(cnt)
    check(fn(exec.handle, C.byref(ls), C.byref(rs), O.pred2(less).id, out.to_col(), _p32(cnt),
             None))
    return out


def set_union(exec: Executor, left, right, less=O.Less) -> DeviceVec:
    """vector::set_union (massively/src/api/algorithm/set.rs:47)."""
    return _set(exec, left, right, less, _L().mb_set_union, len(left) + len(right))


def set_intersection(exec: Executor, left, right, less=O.Less) -> DeviceVec:
    """vector::set_intersection (set.rs:99)."""
    return _set(exec, left, right, less, _L().mb_set_intersection, len(left))


def set_difference(exec: Executor, left, right, less=O.Less) -> DeviceVec:
    """vector::set_difference (set.rs:151)."""
    return _set(exec, left, right, less, _L().mb_set_difference, len(left))
