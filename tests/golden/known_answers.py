"""Known-answer vectors of massively's own tests and doctests, restated.

Each entry cites the test (path inside the massively project) whose inputs
and asserted outputs it carries.  The oracle is pinned against every entry
(tests/test_oracle_golden.py) and the CUDA path is checked against the same
entries (the `test_known_answers*` tests of the tests/test_*_gpu.py files).
No generator script: the values
are the literal inputs and expected outputs of those tests.
"""
import numpy as np

U32 = np.uint32

SCAN = [
    # api/algorithm/scan.rs:91-94 (inclusive_scan, Add)
    dict(src="massively/src/api/algorithm/scan.rs:91-94", kind="inclusive", op="add",
         x=np.array([1, 2, 3, 4], U32), want=np.array([1, 3, 6, 10], U32)),
    # api/algorithm/scan.rs:211-214 (exclusive_scan, init 0)
    dict(src="massively/src/api/algorithm/scan.rs:211-214", kind="exclusive", op="add", init=0,
         x=np.array([1, 2, 3, 4], U32), want=np.array([0, 1, 3, 6], U32)),
    # core/scan.rs:1467-1482 (exclusive applies init once; written into [1..5))
    dict(src="massively/src/core/scan.rs:1467-1482", kind="exclusive", op="add", init=10,
         x=np.array([1, 2, 3, 4], U32), want=np.array([10, 11, 13, 16], U32)),
]

# core/scan.rs:1304-1319: 70,001 ones, probes at block / recursion boundaries.
SCAN_ONES = dict(src="massively/src/core/scan.rs:1304-1319", n=70_001,
                 probes={0: 1, 255: 256, 256: 257, 65_535: 65_536, 70_000: 70_001})
# core/scan.rs:1485-1515: exclusive with init 10 over 70,001 ones, and
# TakeLeft with init 42 over 600 ones -> all 42 (operand order kept).
SCAN_EXCL_ONES = dict(src="massively/src/core/scan.rs:1485-1502", n=70_001, init=10,
                      probes=[0, 255, 256, 65_535, 70_000])
SCAN_TAKE_LEFT = dict(src="massively/src/core/scan.rs:1504-1515", n=600, init=42, want=42)

REDUCE = [
    # api/algorithm/reduce.rs:26-30
    dict(src="massively/src/api/algorithm/reduce.rs:26-30", op="add", init=0,
         x=np.array([1, 2, 3, 4], U32), want=10),
]

SELECT = [
    # api/algorithm/selection.rs:140-144
    dict(src="massively/src/api/algorithm/selection.rs:140-144", kind="copy_where",
         x=np.array([10, 20, 30, 40], U32), stencil=np.array([1, 0, 1, 0], U32),
         want=np.array([10, 30], U32)),
    # api/algorithm/selection.rs:197-201
    dict(src="massively/src/api/algorithm/selection.rs:197-201", kind="remove_where",
         x=np.array([10, 20, 30, 40], U32), stencil=np.array([1, 0, 1, 0], U32),
         want=np.array([20, 40], U32)),
    # core/selection.rs:697-707 (remove_where inverts a non-zero stencil)
    dict(src="massively/src/core/selection.rs:697-707", kind="remove_where",
         x=np.array([10, 20, 30, 40], U32), stencil=np.array([0, 1, 0, 1], U32),
         want=np.array([10, 30], U32)),
    # api/algorithm/selection.rs:466-472
    dict(src="massively/src/api/algorithm/selection.rs:466-472", kind="copy_where",
         x=np.array([10, 20, 30, 40, 50], U32), stencil=np.array([1, 0, 1, 0, 1], U32),
         want=np.array([10, 30, 50], U32)),
]

# core/selection.rs:604-628: three columns (u32, f32, i32), flags [0,1,1,0].
COPY_WHERE_ROWS = dict(
    src="massively/src/core/selection.rs:604-628",
    cols=[np.array([1, 2, 3, 4], U32), np.array([10, 20, 30, 40], np.float32),
          np.array([100, 200, 300, 400], np.int32)],
    stencil=np.array([0, 1, 1, 0], U32),
    want=[np.array([2, 3], U32), np.array([20, 30], np.float32), np.array([200, 300], np.int32)])

# core/selection.rs:631-643: the fused stencil scan of flags [0,7,3,0]
# gives positions [0,1,2,2] (inclusive scan of IsTrue flags).
STENCIL_POSITIONS = dict(src="massively/src/core/selection.rs:631-643",
                         stencil=np.array([0, 7, 3, 0], U32), want=np.array([0, 1, 2, 2], U32))

PARTITION = [
    # core/selection.rs:719-727 (IsEven)
    dict(src="massively/src/core/selection.rs:719-727", pred="is_even",
         x=np.array([3, 2, 4, 1, 6, 5], U32), want=np.array([2, 4, 6, 3, 1, 5], U32),
         boundary=3),
    # api/algorithm/selection.rs:266-270 (Even)
    dict(src="massively/src/api/algorithm/selection.rs:266-270", pred="is_even",
         x=np.array([1, 2, 3, 4], U32), want=np.array([2, 4, 1, 3], U32), boundary=2),
]

GATHER = [
    # api/algorithm/indexed.rs:166-170
    dict(src="massively/src/api/algorithm/indexed.rs:166-170",
         values=np.array([10, 20, 30], U32), idx=np.array([2, 0, 1], U32), stencil=None,
         out=None, want=np.array([30, 10, 20], U32)),
    # api/algorithm/indexed.rs:221-235 (gather_where)
    dict(src="massively/src/api/algorithm/indexed.rs:221-235",
         values=np.array([10, 20, 30], U32), idx=np.array([2, 0, 1], U32),
         stencil=np.array([1, 0, 1], U32), out=np.array([99, 99, 99], U32),
         want=np.array([30, 99, 20], U32)),
    # api/algorithm/indexed.rs:331-345 (an unselected index may be out of range)
    dict(src="massively/src/api/algorithm/indexed.rs:331-345",
         values=np.array([10, 20, 30], U32), idx=np.array([2, 0xFFFFFFFF, 1], U32),
         stencil=np.array([1, 0, 1], U32), out=np.array([99, 99, 99], U32),
         want=np.array([30, 99, 20], U32)),
]

SCATTER = [
    # api/algorithm/scatter.rs:234-246
    dict(src="massively/src/api/algorithm/scatter.rs:234-246",
         values=np.array([10, 20, 30], U32), idx=np.array([2, 0, 1], U32), stencil=None,
         out=np.array([0, 0, 0], U32), want=np.array([20, 30, 10], U32)),
    # api/algorithm/scatter.rs:299-313 (scatter_where)
    dict(src="massively/src/api/algorithm/scatter.rs:299-313",
         values=np.array([10, 20, 30], U32), idx=np.array([2, 0, 1], U32),
         stencil=np.array([1, 0, 1], U32), out=np.array([99, 99, 99], U32),
         want=np.array([99, 30, 10], U32)),
]

REPLACE_WHERE = [
    # api/algorithm/selection.rs:349-361 (doctest)
    dict(src="massively/src/api/algorithm/selection.rs:349-361", value=99,
         stencil=np.array([0, 1, 0, 1], U32), out=np.array([10, 20, 30, 40], U32),
         want=np.array([10, 99, 30, 99], U32)),
    # tests/vector/api/owned.rs:301-310 (value 3 = a reduced total)
    dict(src="massively/tests/vector/api/owned.rs:301-310", value=3,
         stencil=np.array([0, 1, 0], U32), out=np.array([8, 8, 8], U32),
         want=np.array([8, 3, 8], U32)),
]

TRANSFORM_WHERE = [
    # api/algorithm/selection.rs:397-434 (doctest; AddOne)
    dict(src="massively/src/api/algorithm/selection.rs:397-434", op=lambda x: x + 1,
         x=np.array([1, 2, 3], U32), stencil=np.array([1, 0, 1], U32),
         out=np.array([100, 100, 100], U32), want=np.array([2, 100, 4], U32)),
    # tests/vector/api/iter.rs:31-46 (Identity under an all-true stencil)
    dict(src="massively/tests/vector/api/iter.rs:31-46", op=lambda x: x,
         x=np.array([1, 2, 3], U32), stencil=np.array([1, 1, 1], U32),
         out=np.array([0, 0, 0], U32), want=np.array([1, 2, 3], U32)),
]

SORT = [
    # api/algorithm/ordering.rs:59-62
    dict(src="massively/src/api/algorithm/ordering.rs:59-62",
         x=np.array([3, 1, 2], U32), want=np.array([1, 2, 3], U32)),
]

SORT_BY_KEY = [
    # api/algorithm/by_key.rs:214-224
    dict(src="massively/src/api/algorithm/by_key.rs:214-224",
         keys=np.array([3, 1, 2], U32), values=np.array([30, 10, 20], U32),
         want=np.array([10, 20, 30], U32)),
]

RADIX = [
    # api/algorithm/by_key.rs:266-270 (i32 keys, stable)
    dict(src="massively/src/api/algorithm/by_key.rs:266-270",
         keys=[np.array([3, -1, 2, -1], np.int32)], want_perm=None,
         values=np.array([30, 10, 20, 11], U32), want=np.array([10, 11, 20, 30], U32)),
]

# tests/vector/api/radix.rs:25-50: integer extremes; expected = stable order
# by key of the index column.
RADIX_INTEGER_EXTREMES = [
    dict(src="massively/tests/vector/api/radix.rs:45", keys=np.array(
        [0xFFFFFFFF, 0, 1, 1 << 31, 0, 0xFFFFFFFF], U32), want=[1, 4, 2, 3, 0, 5]),
    dict(src="massively/tests/vector/api/radix.rs:46", keys=np.array(
        [0xFFFFFFFFFFFFFFFF, 0, 1, 1 << 63, 0, 0xFFFFFFFFFFFFFFFF], np.uint64),
        want=[1, 4, 2, 3, 0, 5]),
    dict(src="massively/tests/vector/api/radix.rs:47", keys=np.array(
        [2**31 - 1, -2**31, -1, 0, -2**31, 2**31 - 1], np.int32), want=[1, 4, 2, 3, 0, 5]),
    dict(src="massively/tests/vector/api/radix.rs:48", keys=np.array(
        [2**63 - 1, -2**63, -1, 0, -2**63, 2**63 - 1], np.int64), want=[1, 4, 2, 3, 0, 5]),
]


def _f32(bits):
    return np.array(bits, np.uint32).view(np.float32)


def _f64(bits):
    return np.array(bits, np.uint64).view(np.float64)


# tests/vector/api/radix.rs:73-115: float total order (signed NaN payloads,
# +-inf, +-0).  Expected order is f32::total_cmp, stable.
RADIX_FLOAT_TOTAL_ORDER = [
    dict(src="massively/tests/vector/api/radix.rs:94-104", keys=np.concatenate([
        _f32([0x7FC00001]), np.array([np.inf, -0.0, 0.0, -np.inf], np.float32),
        _f32([0xFFC00001]), np.array([1.5, -1.5, -0.0], np.float32)]),
        want=[5, 4, 7, 2, 8, 3, 6, 1, 0]),
    dict(src="massively/tests/vector/api/radix.rs:105-115", keys=np.concatenate([
        _f64([0x7FF8000000000001]), np.array([np.inf, -0.0, 0.0, -np.inf], np.float64),
        _f64([0xFFF8000000000001]), np.array([1.5, -1.5, -0.0], np.float64)]),
        want=[5, 4, 7, 2, 8, 3, 6, 1, 0]),
]

# tests/vector/api/radix.rs:118-162: three compound key columns, seven
# value columns (column*100 + index); expected order by (first, second, third).
RADIX_COMPOUND = dict(
    src="massively/tests/vector/api/radix.rs:118-162",
    keys=[np.array([1, -1, 1, -1, 1, -1, 1, -1, 1], np.int32),
          np.array([2, 2, 1, 2, 1, 1, 1, 1, 1], U32),
          np.array([0, 0, 2, 0, 1, 2, 1, 1, 1], U32)],
    want=[7, 5, 1, 3, 4, 6, 8, 2, 0])

# tests/vector/api/radix.rs:262-275: 513 keys (i*37) % 11, values = index.
RADIX_513 = dict(src="massively/tests/vector/api/radix.rs:262-275", n=513)

BY_KEY = [
    # api/algorithm/by_key.rs:603-616 (reduce_by_key, init 0, Add)
    dict(src="massively/src/api/algorithm/by_key.rs:603-616", kind="reduce",
         keys=np.array([1, 1, 2, 2], U32), values=np.array([10, 20, 30, 40], U32), init=0,
         want_keys=np.array([1, 2], U32), want=np.array([30, 70], U32)),
    # api/algorithm/by_key.rs:386-397 (inclusive_scan_by_key)
    dict(src="massively/src/api/algorithm/by_key.rs:386-397", kind="inclusive",
         keys=np.array([1, 1, 2, 2], U32), values=np.array([10, 20, 30, 40], U32), init=0,
         want=np.array([10, 30, 30, 70], U32)),
    # api/algorithm/by_key.rs:483-495 (exclusive_scan_by_key, init 0)
    dict(src="massively/src/api/algorithm/by_key.rs:483-495", kind="exclusive",
         keys=np.array([1, 1, 2, 2], U32), values=np.array([10, 20, 30, 40], U32), init=0,
         want=np.array([0, 10, 0, 30], U32)),
]

# core/by_key.rs:341-430: 600 rows, keys 1 for i < 300 else 2, seven value
# columns of constants 1..7.  inclusive: column 1 (299, 300, 599) ->
# (300, 1, 300), column 7 -> (2100, 7, 2100); exclusive with inits
# (10..70): column 1 (0, 1, 300, 301) -> (10, 11, 10, 11); reduce with the
# same inits: keys [1, 2], column 1 [310, 310], column 7 [2170, 2170].
BY_KEY_SEVEN = dict(src="massively/src/core/by_key.rs:341-430", n=600,
                    inits=[10, 20, 30, 40, 50, 60, 70])

MERGE = [
    # api/algorithm/merge.rs:103-107
    dict(src="massively/src/api/algorithm/merge.rs:103-107", left=np.array([1, 3, 5], U32),
         right=np.array([2, 4, 6], U32), want=np.array([1, 2, 3, 4, 5, 6], U32)),
]
MERGE_BY_KEY = dict(src="massively/src/api/algorithm/merge.rs:179-193",
                    lk=np.array([1, 3], U32), lv=np.array([10, 30], U32),
                    rk=np.array([2, 4], U32), rv=np.array([20, 40], U32),
                    want=np.array([10, 20, 30, 40], U32))

SETS = [
    # core/set.rs:418-471
    dict(src="massively/src/core/set.rs:418-471", left=np.array([1, 2, 2, 2, 4], U32),
         right=np.array([2, 2, 3, 4, 4], U32), union=np.array([1, 2, 2, 2, 3, 4, 4], U32),
         intersection=np.array([2, 2, 4], U32), difference=np.array([1, 2], U32)),
    # api/algorithm/set.rs:124-192
    dict(src="massively/src/api/algorithm/set.rs:124-192", left=np.array([1, 2, 2, 4], U32),
         right=np.array([2, 3, 4], U32), union=np.array([1, 2, 2, 3, 4], U32),
         intersection=np.array([2, 4], U32), difference=np.array([1, 2], U32)),
]

BOUNDS = [
    # api/algorithm/search.rs doctests of lower_bound and upper_bound
    dict(src="massively/src/api/algorithm/search.rs:75-79, 122-126",
         source=np.array([1, 3, 5, 7], U32), values=np.array([0, 3, 6, 8], U32),
         lower=np.array([0, 1, 3, 4], U32), upper=np.array([0, 2, 3, 4], U32)),
]

UNIQUE = [
    # api/algorithm/ordering.rs:141-144
    dict(src="massively/src/api/algorithm/ordering.rs:141-144",
         x=np.array([1, 1, 2, 2, 3], U32), want=np.array([1, 2, 3], U32)),
]

# Predicates, first-index searches and extrema: the doctests of
# massively/src/api/algorithm/{predicate,ordering,search}.rs and the unit tests
# of massively/src/core/predicate.rs.  `fn` names the vector:: function; `a`
# (and `b`) the inputs; `arg` the predicate (mb_unary name) or order; `want`
# the result (None for massively's None).
PREDICATES = [
    dict(src="massively/src/api/algorithm/predicate.rs:87-89", fn="count_if",
         a=np.array([1, 2, 3, 4], U32), arg="is_even", want=2),
    dict(src="massively/src/api/algorithm/predicate.rs:117-121", fn="all_of",
         a=np.array([2, 4, 6], U32), arg="is_even", want=True),
    dict(src="massively/src/api/algorithm/predicate.rs:149-153", fn="any_of",
         a=np.array([1, 3, 4], U32), arg="is_even", want=True),
    dict(src="massively/src/api/algorithm/predicate.rs:181-185", fn="none_of",
         a=np.array([1, 3, 5], U32), arg="is_even", want=True),
    dict(src="massively/src/api/algorithm/predicate.rs:210-215", fn="find_if",
         a=np.array([1, 3, 4, 6], U32), arg="is_even", want=2),
    dict(src="massively/src/api/algorithm/predicate.rs:256-260", fn="is_partitioned",
         a=np.array([2, 4, 1, 3], U32), arg="is_even", want=True),
    dict(src="massively/src/core/predicate.rs:354-361", fn="count_if",
         a=np.array([7, 0, 3], U32), arg="is_true", want=2),
    dict(src="massively/src/core/predicate.rs:364-376", fn="is_partitioned",
         a=np.array([20, 0], U32), arg="is_even", want=True),
    dict(src="massively/src/core/predicate.rs:424-431", fn="find_if",
         a=np.array([1, 3, 5, 7], U32), arg="is_negative", want=None),
    dict(src="massively/tests/vector/api/runtime.rs:97-99", fn="find_if",
         a=np.array([], U32), arg="is_even", want=None),
    dict(src="massively/src/api/algorithm/ordering.rs:99-105", fn="adjacent_find",
         a=np.array([1, 2, 2, 3], U32), arg="equal", want=1),
    dict(src="massively/src/api/algorithm/ordering.rs:205-210", fn="is_sorted_until",
         a=np.array([1, 2, 4, 3, 5], U32), arg="less", want=3),
    dict(src="massively/src/api/algorithm/ordering.rs:249-253", fn="is_sorted",
         a=np.array([1, 2, 3, 4], U32), arg="less", want=True),
    dict(src="massively/src/api/algorithm/ordering.rs:315-321", fn="min_element",
         a=np.array([3, 1, 2, 1], U32), arg="less", want=1),
    dict(src="massively/src/api/algorithm/ordering.rs:348-354", fn="max_element",
         a=np.array([3, 1, 3, 2], U32), arg="less", want=0),
    dict(src="massively/src/api/algorithm/ordering.rs:404-410", fn="minmax_element",
         a=np.array([3, 1, 4, 2], U32), arg="less", want=(1, 2)),
    dict(src="massively/src/api/algorithm/search.rs:26-31", fn="find_first_of",
         a=np.array([1, 2, 3, 4], U32), b=np.array([7, 3], U32), arg="equal", want=2),
    dict(src="massively/src/api/algorithm/search.rs:167-172", fn="equal",
         a=np.array([1, 2, 3], U32), b=np.array([1, 2, 3], U32), arg="equal", want=True),
    dict(src="massively/src/api/algorithm/search.rs:223-229", fn="mismatch",
         a=np.array([1, 2, 3], U32), b=np.array([1, 4, 3], U32), arg="equal", want=1),
    dict(src="massively/src/api/algorithm/search.rs:281-286", fn="lexicographical_compare",
         a=np.array([1, 2, 3], U32), b=np.array([1, 3, 0], U32), arg="less", want=True),
]

# scatter_reduce: the doctest of massively/src/api/algorithm/scatter.rs and
# its unit tests (multi-column rows, component-wise add).  `values` /
# `output` are lists of columns; `want` the outputs after the call.
SCATTER_REDUCE = [
    dict(src="massively/src/api/algorithm/scatter.rs:361-375",
         values=[np.array([2, 3, 5, 7], U32)], indices=np.array([1, 0, 1, 1], U32),
         init=[0], op="add", output=[np.array([10, 20, 30], U32)],
         want=[np.array([13, 34, 30], U32)]),
    dict(src="massively/src/api/algorithm/scatter.rs:447-466",
         values=[np.array([1, 2, 3], U32), np.array([10, 20, 30], U32)],
         indices=np.array([1, 0, 1], U32), init=[0, 0], op="add",
         output=[np.array([100, 200], U32), np.array([1000, 2000], U32)],
         want=[np.array([102, 204], U32), np.array([1020, 2040], U32)]),
    dict(src="massively/src/api/algorithm/scatter.rs:469-495",
         values=[np.array([1, 2, 3], U32), np.array([10, 20, 30], U32),
                 np.array([100, 200, 300], U32)],
         indices=np.array([1, 0, 1], U32), init=[0, 0, 0], op="add",
         output=[np.array([100, 200], U32), np.array([1000, 2000], U32),
                 np.array([10000, 20000], U32)],
         want=[np.array([102, 204], U32), np.array([1020, 2040], U32),
               np.array([10200, 20400], U32)]),
]

# Per-segment queries: massively/tests/seg/api.rs.  `query` is the
# ForEachSegment algorithm, `want` one u32 per segment (flags as 0 / 1).
SEG_QUERIES = [
    dict(src="massively/tests/seg/api.rs:718-741", query="all_of", op="is_even",
         x=np.array([2, 4, 3, 6], U32), offsets=np.array([0, 2, 4], U32),
         want=np.array([1, 0], U32)),
    dict(src="massively/tests/seg/api.rs:744-762", query="all_of", op="is_true",
         x=np.array([7, 3, 0], U32), offsets=np.array([0, 2, 3], U32),
         want=np.array([1, 0], U32)),
    dict(src="massively/tests/seg/api.rs:766-805", query="find_if", op="is_even",
         x=np.array([2, 4, 6, 1, 1, 3, 5, 7, 8, 8], U32),
         offsets=np.array([0, 0, 3, 6, 7, 10], U32), want=np.array([0, 0, 3, 1, 1], U32)),
    dict(src="massively/tests/seg/api.rs:807-813", query="adjacent_find", op="equal",
         x=np.array([2, 4, 6, 1, 1, 3, 5, 7, 8, 8], U32),
         offsets=np.array([0, 0, 3, 6, 7, 10], U32), want=np.array([0, 3, 0, 1, 1], U32)),
]

# ForEachSegment(Take(k)): massively/tests/seg/api.rs:771-797 -- values and
# new offsets, empty segments included.
SEG_TAKE = [
    dict(src="massively/tests/seg/api.rs:771-784", k=2,
         x=np.array([2, 4, 6, 1, 1, 3, 5, 7, 8, 8], U32),
         offsets=np.array([0, 0, 3, 6, 7, 10], U32),
         values=np.array([2, 4, 1, 1, 5, 7, 8], U32), new_offsets=np.array([0, 0, 2, 4, 5, 7], U32)),
    dict(src="massively/tests/seg/api.rs:786-797", k=0,
         x=np.array([2, 4, 6, 1, 1, 3, 5, 7, 8, 8], U32),
         offsets=np.array([0, 0, 3, 6, 7, 10], U32),
         values=np.array([], U32), new_offsets=np.array([0, 0, 0, 0, 0, 0], U32)),
]

# massively/tests/vector/api/predicate.rs:17-22: count_if over a lazy
# counting view of four billion items (u32 lengths above i32::MAX).
COUNT_IF_FOUR_BILLION = dict(src="massively/tests/vector/api/predicate.rs:17-22",
                             n=4_000_000_000, pred="is_even", want=2_000_000_000)

SEG = [
    # tests/seg/api.rs:288-322: Reduce(Add, 0) over offsets [0,3,5]
    dict(src="massively/tests/seg/api.rs:288-322", kind="reduce", op="add", init=0,
         x=np.array([1, 1, 2, 3, 3], U32), offsets=np.array([0, 3, 5], U32),
         want=np.array([4, 6], U32)),
    # tests/seg/api.rs:330-347: ExclusiveScan(Add, 0) and Reduce(Add, 0)
    dict(src="massively/tests/seg/api.rs:330-339", kind="exclusive", op="add", init=0,
         x=np.array([1, 2, 4], U32), offsets=np.array([0, 2, 3], U32),
         want=np.array([0, 1, 0], U32)),
    dict(src="massively/tests/seg/api.rs:341-347", kind="reduce", op="add", init=0,
         x=np.array([1, 2, 4], U32), offsets=np.array([0, 2, 3], U32),
         want=np.array([3, 4], U32)),
    # tests/seg/api.rs:626-659: lengths [2,0,1] -> offsets [0,2,2,3]; the
    # per-entry totals (value + context) [11, 12, 33] reduce to [23, 0, 33]
    # before the empty-segment contribution is added.
    dict(src="massively/tests/seg/api.rs:626-659", kind="reduce", op="add", init=0,
         x=np.array([11, 12, 33], U32), offsets=np.array([0, 2, 2, 3], U32),
         want=np.array([23, 0, 33], U32)),
]

SEGMENTATION = [
    # tests/seg/api.rs:378-394 (from_lengths [1,2,3])
    dict(src="massively/tests/seg/api.rs:378-394", lengths=np.array([1, 2, 3], U32),
         offsets=np.array([0, 1, 3, 6], U32), ids=np.array([0, 1, 1, 2, 2, 2], U32),
         local=np.array([0, 0, 1, 0, 1, 2], U32)),
    # tests/seg/api.rs:415-418 (constant(2).take(3))
    dict(src="massively/tests/seg/api.rs:415-418", lengths=np.array([2, 2, 2], U32),
         offsets=np.array([0, 2, 4, 6], U32), ids=np.array([0, 0, 1, 1, 2, 2], U32),
         local=np.array([0, 1, 0, 1, 0, 1], U32)),
    # tests/seg/api.rs:425-435 (empty segments)
    dict(src="massively/tests/seg/api.rs:425-435", lengths=np.array([1, 0, 2, 0], U32),
         offsets=np.array([0, 1, 1, 3, 3], U32), ids=np.array([0, 2, 2], U32),
         local=np.array([0, 0, 1], U32)),
    # tests/seg/api.rs:445-449 (no segments)
    dict(src="massively/tests/seg/api.rs:445-449", lengths=np.array([], U32),
         offsets=np.array([0], U32), ids=np.array([], U32), local=np.array([], U32)),
]

# tests/seg/api.rs:509-515: invalid offsets.
INVALID_OFFSETS = dict(src="massively/tests/seg/api.rs:509-515",
                       cases=[np.array([], U32), np.array([1, 1], U32),
                              np.array([0, 2, 1], U32)])
# tests/seg/api.rs:534-538: lengths overflowing u32.
OVERFLOWING_LENGTHS = dict(src="massively/tests/seg/api.rs:534-538",
                           lengths=np.array([0xFFFFFFFF, 1], U32))

# verification/oracle/tests/vector/common.rs:12-14 and tests/seg.rs:20-28
ORACLE_LENGTHS = [0, 1, 2, 31, 32, 33, 255, 256, 257, 511, 512, 513, 767, 768, 769, 1023,
                  1024, 1025]
SEGMENT_LENGTHS = [0, 1, 2, 31, 32, 33, 127, 128, 129, 255, 256, 257]
