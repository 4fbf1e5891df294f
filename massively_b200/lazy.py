"""Lazy views evaluated inside the consuming kernel's loads.

Mirrors massively/src/api/lazy.rs:664-922.  A view whose child is a device
column lowers to one mb_src descriptor that the kernel evaluates per item
(column, constant, counting, stride, permute, reverse, repeat_each, tile,
plus a built-in unary map on top).  A deeper tree is lowered by first
materialising its inner views with `mb_copy` (one fused kernel per level).
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from . import op as O
from .runtime import ID_TO_NP, NP_TO_ID, DeviceVec, Executor, check, value_bits

U32 = np.dtype(np.uint32)


class View:
    """Base of lazy views: `len`, the produced element type `dtype`."""

    len: int
    dtype: np.dtype

    def __len__(self):
        return self.len

    def lower(self, exec: Executor, keep: list) -> N.mb_src:  # pragma: no cover - abstract
        raise NotImplementedError

    def take(self, n: int) -> "View":
        v = _copy_view(self)
        v.len = int(n)
        return v


def _copy_view(v):
    import copy
    return copy.copy(v)


def lower(exec: Executor, x, keep: list) -> N.mb_src:
    """mb_src for a DeviceVec or a View (keeps temporaries alive in `keep`)."""
    if isinstance(x, DeviceVec):
        return x.to_src()
    if isinstance(x, View):
        return x.lower(exec, keep)
    raise TypeError(f"not a device column or lazy view: {type(x).__name__}")


def _as_column(exec: Executor, x, keep: list) -> DeviceVec:
    """A device column for `x` (materialised when it is a view)."""
    if isinstance(x, DeviceVec):
        return x
    s = lower(exec, x, keep)
    out = exec.alloc(ID_TO_NP[s.vtype], s.len)
    check(N.lib().mb_copy(exec.handle, s, out.to_col()))
    keep.append(out)
    return out


def dtype_of(x) -> np.dtype:
    return x.dtype


class Constant(View):
    """lazy::constant(value).take(n)."""

    def __init__(self, value, dtype=None, n: int = 0):
        self.value = value
        self.dtype = np.dtype(dtype) if dtype is not None else np.asarray(value).dtype
        self.len = n

    def lower(self, exec, keep):
        s = N.mb_src()
        s.kind = N.SRC_CONSTANT
        s.dtype = s.vtype = NP_TO_ID[self.dtype]
        s.a = value_bits(self.value, self.dtype)
        s.len = self.len
        return s


class Counting(View):
    """lazy::counting(start).take(n): start, start+1, ... (MIndex)."""

    def __init__(self, start: int = 0, n: int = 0, dtype=U32):
        self.start, self.len, self.dtype = int(start), n, np.dtype(dtype)

    def lower(self, exec, keep):
        s = N.mb_src()
        s.kind = N.SRC_COUNTING
        s.dtype = s.vtype = NP_TO_ID[self.dtype]
        s.a = value_bits(self.start, self.dtype)
        s.len = self.len
        return s


class Stride(View):
    """lazy::stride(start, step).take(n)."""

    def __init__(self, start: int, step: int, n: int = 0, dtype=U32):
        self.start, self.step, self.len, self.dtype = int(start), int(step), n, np.dtype(dtype)

    def lower(self, exec, keep):
        s = N.mb_src()
        s.kind = N.SRC_STRIDE
        s.dtype = s.vtype = NP_TO_ID[self.dtype]
        s.a = value_bits(self.start, self.dtype)
        s.b = value_bits(self.step, self.dtype)
        s.len = self.len
        return s


class _Unary(View):
    """A view over one child column: permute / reverse / repeat_each / tile."""

    kind = N.SRC_COLUMN

    def __init__(self, values, n: int, a: int = 0, index=None):
        self.values, self.len, self.a, self.index = values, n, a, index
        self.dtype = values.dtype

    def lower(self, exec, keep):
        col = _as_column(exec, self.values, keep)
        s = col.to_src()
        s.kind = self.kind
        s.len = self.len
        s.a = self.a
        s.len_dev = None
        if self.index is not None:
            idx = _as_column(exec, self.index, keep)
            s.index = idx.data_ptr() if len(idx) else None
        return s


class Permute(_Unary):
    kind = N.SRC_PERMUTE


class Reverse(_Unary):
    kind = N.SRC_REVERSE


class RepeatEach(_Unary):
    kind = N.SRC_REPEAT_EACH


class Tile(_Unary):
    kind = N.SRC_TILE


class Map(View):
    """lazy::map(input, op): a built-in unary op (or a cast) on each read."""

    def __init__(self, values, unary, dtype=None):
        self.values, self.op = values, O.unary(unary)
        if dtype is not None:
            self.dtype = np.dtype(dtype)
        elif self.op.is_predicate:
            self.dtype = U32
        else:
            self.dtype = values.dtype
        self.len = len(values)

    def lower(self, exec, keep):
        inner = self.values
        if isinstance(inner, Map) and inner.op.id != 0:
            inner = _as_column(exec, inner, keep)
        if isinstance(inner, Map):  # identity / cast under this map
            inner = _as_column(exec, inner, keep)
        s = lower(exec, inner, keep)
        if s.map != 0:
            col = _as_column(exec, inner, keep)
            s = col.to_src()
        s.map = self.op.id
        s.vtype = NP_TO_ID[self.dtype]
        s.len = self.len
        return s


class AdjacentDifference(View):
    """lazy::adjacent_difference(input, op): out[0] = x[0], out[i] =
    op(x[i-1], x[i]), evaluated inside the consuming kernel's load
    (MB_SRC_ADJACENT)."""

    def __init__(self, values, reduction):
        self.values, self.op = values, O.reduction(reduction)
        self.dtype, self.len = values.dtype, len(values)

    def lower(self, exec, keep):
        col = _as_column(exec, self.values, keep)
        s = col.to_src()
        s.kind = N.SRC_ADJACENT
        s.b = self.op.id
        s.len = self.len
        s.len_dev = None
        return s


def constant(value, dtype=None) -> Constant:
    return Constant(value, dtype)


def counting(start: int = 0) -> Counting:
    return Counting(start)


def stride(start: int, step: int) -> Stride:
    return Stride(start, step)


def permute(values, indices) -> Permute:
    return Permute(values, len(indices), index=indices)


def reverse(values) -> Reverse:
    return Reverse(values, len(values))


def repeat_each(values, repeats: int) -> RepeatEach:
    return RepeatEach(values, len(values) * int(repeats), a=int(repeats))


def tile(values, repeats: int) -> Tile:
    return Tile(values, len(values) * int(repeats), a=len(values))


def map(values, unary, dtype=None) -> Map:  # noqa: A001 - massively's name
    return Map(values, unary, dtype)


def identity(values) -> Map:
    return Map(values, O.Identity)


def cast(values, dtype) -> Map:
    return Map(values, O.Identity, dtype)


def adjacent_difference(values, reduction) -> AdjacentDifference:
    return AdjacentDifference(values, reduction)
