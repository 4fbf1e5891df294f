"""`seg::*`: Segmentation and per-segment algorithms over the C ABI.

Mirrors massively/src/seg/segmentation.rs:129-441 (Segmentation: offsets are
canonical, validated with one synchronisation) and massively/src/seg/
mod.rs:159-243 (ForEachSegment(algorithm).run(exec, segments)).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from . import op as O
from .lazy import lower
from .runtime import (DeviceVec, Executor, ForeignExecutor, InvalidSegmentation, LengthMismatch,
                      LengthTooLarge, MINDEX_MAX, check, scalar_buffer)

_L = N.lib
U32 = np.dtype(np.uint32)


class Segmentation:
    """A validated partition of a flat value range into ordered segments."""

    def __init__(self, offsets: DeviceVec, value_count: int):
        self._offsets = offsets
        self._value_count = int(value_count)

    @classmethod
    def from_offsets(cls, exec: Executor, offsets) -> "Segmentation":
        """Segmentation::from_offsets (segmentation.rs:196-232)."""
        off = _u32_column(exec, offsets)
        if len(off) == 0:
            raise InvalidSegmentation()
        vc = C.c_uint32(0)
        check(_L().mb_segmentation_validate_offsets(exec.handle, C.c_void_p(off.data_ptr()),
                                                    len(off), C.byref(vc)))
        return cls(off, vc.value)

    @classmethod
    def from_lengths(cls, exec: Executor, lengths) -> "Segmentation":
        """Segmentation::from_lengths (segmentation.rs:238-280)."""
        n = len(lengths)
        if n >= MINDEX_MAX:
            raise LengthTooLarge(n + 1)
        keep = []
        s = lower(exec, lengths, keep) if n else None
        off = exec.alloc(U32, n + 1)
        if n == 0:
            off.tensor.zero_()
            return cls(off, 0)
        vc = C.c_uint32(0)
        check(_L().mb_segmentation_from_lengths(exec.handle, C.byref(s),
                                                C.c_void_p(off.data_ptr()), C.byref(vc)))
        return cls(off, vc.value)

    @classmethod
    def from_segment_ids(cls, exec: Executor, ids, segment_count: int) -> "Segmentation":
        """Segmentation::from_segment_ids (segmentation.rs:290-335): ids must be
        non-decreasing and < segment_count."""
        if segment_count >= MINDEX_MAX:
            raise LengthTooLarge(segment_count + 1)
        keep = []
        s = lower(exec, ids, keep)
        off = exec.alloc(U32, segment_count + 1)
        check(_L().mb_segmentation_from_segment_ids(exec.handle, C.byref(s), segment_count,
                                                    C.c_void_p(off.data_ptr())))
        return cls(off, len(ids))

    def offsets(self) -> DeviceVec:
        return self._offsets

    def segment_count(self) -> int:
        return len(self._offsets) - 1

    def value_count(self) -> int:
        return self._value_count

    def lengths(self, exec: Executor) -> DeviceVec:
        """Segmentation::lengths: one length per segment."""
        out = exec.alloc(U32, self.segment_count())
        if self.segment_count():
            check(_L().mb_segmentation_lengths(exec.handle, C.c_void_p(self._offsets.data_ptr()),
                                               self.segment_count(), C.c_void_p(out.data_ptr())))
        return out

    def segment_ids(self, exec: Executor) -> DeviceVec:
        """Segmentation::segment_ids: flat value -> segment index."""
        out = exec.alloc(U32, self._value_count)
        if self._value_count:
            check(_L().mb_segmentation_segment_ids(
                exec.handle, C.c_void_p(self._offsets.data_ptr()), self.segment_count(),
                C.c_void_p(out.data_ptr()), self._value_count))
        return out

    def local_indices(self, exec: Executor) -> DeviceVec:
        """Segmentation::local_indices: position of each value in its segment."""
        out = exec.alloc(U32, self._value_count)
        if self._value_count:
            check(_L().mb_segmentation_local_indices(
                exec.handle, C.c_void_p(self._offsets.data_ptr()), self.segment_count(),
                C.c_void_p(out.data_ptr()), self._value_count))
        return out

    def segments(self, values) -> "SegmentIterator":
        if len(values) != self._value_count:
            raise LengthMismatch(self._value_count, len(values))
        return SegmentIterator(values, self)


class SegmentIterator:
    """Values paired with their segmentation (seg/mod.rs:49-99)."""

    def __init__(self, values, segmentation: Segmentation):
        self._values, self._seg = values, segmentation

    def values(self):
        return self._values

    def offsets(self) -> DeviceVec:
        return self._seg.offsets()

    def segmentation(self) -> Segmentation:
        return self._seg


def _u32_column(exec: Executor, x) -> DeviceVec:
    from .lazy import _as_column
    keep = []
    col = _as_column(exec, x, keep)
    if col.dtype != U32:
        raise LengthMismatch(4, col.dtype.itemsize)
    if col.owner != exec.id:
        raise ForeignExecutor()
    return col


# --------------------------------------------------------- algorithms ------

class InclusiveScan:
    def __init__(self, op):
        self.op = O.reduction(op)


class ExclusiveScan:
    def __init__(self, op, init):
        self.op, self.init = O.reduction(op), init


class Reduce:
    def __init__(self, op, init):
        self.op, self.init = O.reduction(op), init


class Sort:
    def __init__(self, less=O.Less):
        self.less = O.pred2(less)


class _Query:
    """A per-segment query: one u32 per segment (seg/mod.rs:211-245)."""
    query = -1

    def __init__(self, op):
        self.op = op

    def op_id(self) -> int:
        return O.unary(self.op).id


class CountIf(_Query):
    """Items the predicate passes."""
    query = 0


class FindIf(_Query):
    """First passing local index, or the segment's length."""
    query = 1


class AdjacentFind(_Query):
    """First local i with x[i] == x[i+1], or the segment's length."""
    query = 2

    def __init__(self, equal=O.Equal):
        super().__init__(equal)

    def op_id(self) -> int:
        return O.pred2(self.op).id


class IsSortedUntil(_Query):
    """First local i with less(x[i], x[i-1]), or the segment's length."""
    query = 3

    def __init__(self, less=O.Less):
        super().__init__(less)

    def op_id(self) -> int:
        return O.pred2(self.op).id


class AllOf(_Query):
    query = 4


class AnyOf(_Query):
    query = 5


class NoneOf(_Query):
    query = 6


class IsSorted(IsSortedUntil):
    query = 7


class Map:
    """Map(unary): the same segments over mapped values (seg/mod.rs:165)."""

    def __init__(self, unary, dtype=None):
        self.unary, self.dtype = unary, dtype


class Reverse:
    """Every segment reversed (seg/mod.rs:177)."""


class AdjacentDifference:
    """First item kept, then op(x[i-1], x[i]) inside each segment
    (seg/mod.rs:191)."""

    def __init__(self, op):
        self.op = O.reduction(op)


class _Keep:
    kind = -1

    def param(self) -> int:
        raise NotImplementedError


class Filter(_Keep):
    """The items the predicate passes, per segment (seg/mod.rs:199)."""
    kind = 0

    def __init__(self, pred):
        self.pred = O.unary(pred)

    def param(self) -> int:
        return self.pred.id


class Take(_Keep):
    """The first k items of every segment (seg/mod.rs:203)."""
    kind = 1

    def __init__(self, count: int):
        self.count = int(count)

    def param(self) -> int:
        return self.count


class Unique(_Keep):
    """The first item of every run of equal items, per segment
    (seg/mod.rs:195)."""
    kind = 2

    def __init__(self, equal=O.Equal):
        self.equal = O.pred2(equal)

    def param(self) -> int:
        return self.equal.id


class ForEachSegment:
    """ForEachSegment(algorithm).run(exec, segments) (seg/mod.rs:159-243).
    Scans and sorts return a SegmentIterator over new values with the same
    offsets; Reduce returns one value per segment (empty -> init)."""

    def __init__(self, algorithm):
        self.algorithm = algorithm

    def run(self, exec: Executor, segments: SegmentIterator):
        a = self.algorithm
        values, sgm = segments.values(), segments.segmentation()
        keep = []
        s = lower(exec, values, keep)
        off = C.c_void_p(sgm.offsets().data_ptr())
        nseg = sgm.segment_count()
        dt = values.dtype
        if isinstance(a, InclusiveScan):
            out = exec.alloc(dt, len(values))
            check(_L().mb_seg_inclusive_scan(exec.handle, C.byref(s), off, nseg, a.op.id,
                                             out.to_col()))
            return SegmentIterator(out, sgm)
        if isinstance(a, ExclusiveScan):
            out = exec.alloc(dt, len(values))
            buf = scalar_buffer(a.init, dt)
            check(_L().mb_seg_exclusive_scan(exec.handle, C.byref(s), off, nseg, a.op.id, buf,
                                             out.to_col()))
            return SegmentIterator(out, sgm)
        if isinstance(a, Reduce):
            out = exec.alloc(dt, nseg)
            buf = scalar_buffer(a.init, dt)
            check(_L().mb_seg_reduce(exec.handle, C.byref(s), off, nseg, a.op.id, buf,
                                     out.to_col()))
            return out
        if isinstance(a, Sort):
            out = exec.alloc(dt, len(values))
            check(_L().mb_seg_sort(exec.handle, C.byref(s), off, nseg, a.less.id, out.to_col()))
            return SegmentIterator(out, sgm)
        if isinstance(a, Map):
            from . import vector
            return SegmentIterator(vector.map(exec, values, a.unary, a.dtype), sgm)
        if isinstance(a, (Reverse, AdjacentDifference)):
            out = exec.alloc(dt, len(values))
            if isinstance(a, Reverse):
                check(_L().mb_seg_reverse(exec.handle, C.byref(s), off, nseg, out.to_col()))
            else:
                check(_L().mb_seg_adjacent_difference(exec.handle, C.byref(s), off, nseg,
                                                      a.op.id, out.to_col()))
            return SegmentIterator(out, sgm)
        if isinstance(a, _Keep):
            out = exec.alloc(dt, len(values))
            new_off = exec.alloc(U32, nseg + 1)
            cnt = C.c_uint32(0)
            check(_L().mb_seg_keep(exec.handle, C.byref(s), off, nseg, a.kind, a.param(),
                                   out.to_col(), C.c_void_p(new_off.data_ptr()), None,
                                   C.byref(cnt)))
            return SegmentIterator(out.slice(0, cnt.value), Segmentation(new_off, cnt.value))
        if isinstance(a, _Query):
            out = exec.alloc(np.uint32, nseg)
            check(_L().mb_seg_query(exec.handle, C.byref(s), off, nseg, a.query, a.op_id(),
                                    out.to_col()))
            return out
        raise TypeError(f"unsupported segment algorithm {type(a).__name__}")
