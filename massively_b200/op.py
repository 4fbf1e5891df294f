"""Built-in operators: the compile-time `op::*` traits of massively, as ids.

massively lets users write `#[cube]` operators (ReductionOp, UnaryOp,
PredicateOp, BinaryPredicateOp: massively/src/core/op.rs:33-96,
massively/src/core/reduce.rs:63-66, massively/src/core/ordering/mod.rs:53-56);
this library compiles a fixed set of them into its kernels
(include/massively_b200.h mb_op / mb_unary / mb_pred2).
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class ReductionOp:
    id: int
    name: str
    commutative: bool = True


@dataclass(frozen=True)
class UnaryOp:
    id: int
    name: str
    is_predicate: bool = False


@dataclass(frozen=True)
class BinaryPredicateOp:
    id: int
    name: str


Add = ReductionOp(0, "add")
Mul = ReductionOp(1, "mul")
Min = ReductionOp(2, "min")
Max = ReductionOp(3, "max")
BitAnd = ReductionOp(4, "and")
BitOr = ReductionOp(5, "or")
BitXor = ReductionOp(6, "xor")
TakeLeft = ReductionOp(7, "take_left", commutative=False)
TakeRight = ReductionOp(8, "take_right", commutative=False)
REDUCTIONS = {o.name: o for o in (Add, Mul, Min, Max, BitAnd, BitOr, BitXor, TakeLeft, TakeRight)}

Identity = UnaryOp(0, "identity")
IsTrue = UnaryOp(1, "is_true", True)
IsFalse = UnaryOp(2, "is_false", True)
IsEven = UnaryOp(3, "is_even", True)
IsOdd = UnaryOp(4, "is_odd", True)
Negate = UnaryOp(5, "negate")
BitNot = UnaryOp(6, "bit_not")
Abs = UnaryOp(7, "abs")
IsNegative = UnaryOp(8, "is_negative", True)
IsPositive = UnaryOp(9, "is_positive", True)
UNARIES = {o.name: o for o in (Identity, IsTrue, IsFalse, IsEven, IsOdd, Negate, BitNot, Abs,
                               IsNegative, IsPositive)}

Less = BinaryPredicateOp(0, "less")
Greater = BinaryPredicateOp(1, "greater")
TotalLess = BinaryPredicateOp(2, "total_less")
Equal = BinaryPredicateOp(3, "equal")
PREDICATES2 = {o.name: o for o in (Less, Greater, TotalLess, Equal)}


def reduction(op) -> ReductionOp:
    return REDUCTIONS[op] if isinstance(op, str) else op


def unary(op) -> UnaryOp:
    return UNARIES[op] if isinstance(op, str) else op


def pred2(op) -> BinaryPredicateOp:
    return PREDICATES2[op] if isinstance(op, str) else op


# ---------------------------------------------------------- user operators --

class UserOp:
    """An operator written as CUDA C source and compiled at run time (NVRTC)
    -- the counterpart of a user `#[cube]` impl of op::ReductionOp /
    op::UnaryOp (massively/src/core/op.rs:33-96).

    binary(exec, dtype, source, name): `source` defines
    `__device__ T name(T a, T b)` (T is the element type); usable with
    vector.reduce (associative and commutative) and the scans (associative).
    map(exec, in_dtype, out_dtype, source, name): `source` defines
    `__device__ Out name(In x)`; usable with vector.map."""

    def __init__(self, handle, kind: int, dtype, out_dtype):
        self.handle, self.kind = handle, kind
        self.dtype, self.out_dtype = dtype, out_dtype
        self.is_predicate = False

    @classmethod
    def binary(cls, exec, dtype, source: str, name: str) -> "UserOp":
        import ctypes as C
        import numpy as np
        from . import _native as N
        from .runtime import NP_TO_ID, check
        h = C.c_void_p()
        dt = np.dtype(dtype)
        check(N.lib().mb_user_op_compile(exec.handle, NP_TO_ID[dt], source.encode(),
                                         name.encode(), C.byref(h)))
        return cls(h, 0, dt, dt)

    @classmethod
    def map(cls, exec, in_dtype, out_dtype, source: str, name: str) -> "UserOp":
        import ctypes as C
        import numpy as np
        from . import _native as N
        from .runtime import NP_TO_ID, check
        h = C.c_void_p()
        i, o = np.dtype(in_dtype), np.dtype(out_dtype)
        check(N.lib().mb_user_map_compile(exec.handle, NP_TO_ID[i], NP_TO_ID[o], source.encode(),
                                          name.encode(), C.byref(h)))
        return cls(h, 1, i, o)

    @classmethod
    def predicate(cls, exec, dtype, source: str, name: str) -> "UserOp":
        """A comparator (op::BinaryPredicateOp): `source` defines
        `__device__ bool name(T a, T b)`, a strict weak order; usable with
        vector.sort and vector.sort_by_key (stable)."""
        import ctypes as C
        import numpy as np
        from . import _native as N
        from .runtime import NP_TO_ID, check
        h = C.c_void_p()
        dt = np.dtype(dtype)
        check(N.lib().mb_user_pred_compile(exec.handle, NP_TO_ID[dt], source.encode(),
                                           name.encode(), C.byref(h)))
        return cls(h, 2, dt, dt)

    @staticmethod
    def check_source(kind: int, dtype, out_dtype, source: str, name: str) -> None:
        """Compiles without loading (no device needed); raises on an error."""
        import numpy as np
        from . import _native as N
        from .runtime import NP_TO_ID, check
        check(N.lib().mb_user_op_check(kind, NP_TO_ID[np.dtype(dtype)],
                                       NP_TO_ID[np.dtype(out_dtype)], source.encode(),
                                       name.encode()))

    def __del__(self):
        try:
            from . import _native as N
            if self.handle:
                N.lib().mb_user_op_destroy(self.handle)
                self.handle = None
        except Exception:  # interpreter shutdown
            pass
