"""Per-segment queries (CountIf, FindIf, AdjacentFind, AllOf, AnyOf, NoneOf,
IsSorted, IsSortedUntil): the CUDA path against the oracle (restating
massively's verification/oracle/src/seg.rs:171-283), exactly, on the
reference's seg API tests and on lognormal segmentations with empty, single
and very long segments, hits planted at 128-item round edges, every element
type and order, and lazy values."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu

QUERIES = {"count_if": "CountIf", "find_if": "FindIf", "all_of": "AllOf", "any_of": "AnyOf",
           "none_of": "NoneOf"}


@pytest.fixture(scope="module")
def ex():
    return executor()


def _run(ex, values, offsets_host, query, op):
    from massively_b200 import op as O, seg
    sgm = seg.Segmentation.from_offsets(ex, ex.to_device(offsets_host))
    it = seg.SegmentIterator(values, sgm)
    if query in QUERIES:
        alg = getattr(seg, QUERIES[query])(op)
    elif query == "adjacent_find":
        alg = seg.AdjacentFind()
    else:
        less = {"less": O.Less, "greater": O.Greater, "total_less": O.TotalLess}[op]
        alg = seg.IsSorted(less) if query == "is_sorted" else seg.IsSortedUntil(less)
    return ex.to_host(seg.ForEachSegment(alg).run(ex, it))


def test_known_answers(ex):
    for case in K.SEG_QUERIES:
        got = _run(ex, ex.to_device(case["x"]), case["offsets"], case["query"], case["op"])
        np.testing.assert_array_equal(got, case["want"], err_msg=case["src"])


def _lognormal_offsets(nseg, seed, scale=40.0):
    rng = np.random.default_rng(seed)
    lens = np.floor(rng.lognormal(1.5, 1.6, nseg) * scale / 10).astype(np.int64)
    lens[rng.integers(0, nseg, max(1, nseg // 10))] = 0  # empty segments
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)


@pytest.mark.parametrize("nseg", [1, 7, 1000, 100_003])
@pytest.mark.parametrize("query", ["count_if", "find_if", "all_of", "any_of", "none_of"])
def test_predicate_queries_u32(ex, nseg, query):
    off = _lognormal_offsets(nseg, nseg)
    n = int(off[-1])
    x = (seeded(np.uint32, n, nseg + 1) | 1).astype(np.uint32)  # odd: fails is_even
    rng = np.random.default_rng(3)
    x[rng.integers(0, max(n, 1), n // 50)] = 4 if n else 0  # sparse passing items
    d = ex.to_device(x)
    for pred in ("is_even", "is_odd"):
        np.testing.assert_array_equal(_run(ex, d, off, query, pred),
                                      orc.seg_query(x, off, query, pred), err_msg=pred)


@pytest.mark.parametrize("dtype", [np.int8, np.uint16, np.int32, np.uint64, np.int64,
                                   np.float32, np.float64])
@pytest.mark.parametrize("query", ["adjacent_find", "is_sorted_until", "is_sorted", "find_if",
                                   "count_if"])
def test_queries_types(ex, dtype, query):
    off = _lognormal_offsets(20_000, 5)
    n = int(off[-1])
    rng = np.random.default_rng(9)
    x = np.sort(rng.integers(-40, 40, n)).astype(dtype) if query.startswith("is_sorted") else \
        rng.integers(-3, 4, n).astype(dtype)
    if query.startswith("is_sorted"):
        x[rng.integers(0, n, n // 500)] = 0  # some descents
    d = ex.to_device(x)
    if query in ("adjacent_find",):
        ops = ["equal"]
    elif query.startswith("is_sorted"):
        ops = ["less", "greater", "total_less"]
    else:
        ops = ["is_negative", "is_positive", "is_true"]
    for op in ops:
        np.testing.assert_array_equal(_run(ex, d, off, query, op),
                                      orc.seg_query(x, off, query, op), err_msg=op)


@pytest.mark.parametrize("query", ["find_if", "adjacent_find", "is_sorted_until", "count_if"])
def test_long_segments_and_round_edges(ex, query):
    """Single segments of up to 2^21 items, hits at 128-item round edges."""
    for length in (127, 128, 129, 4096, 1 << 21):
        for hit in (None, 0, 127, 128, length - 1):
            off = np.array([0, 5, 5 + length, 5 + length + 3], np.uint32)
            n = int(off[-1])
            x = np.arange(n, dtype=np.uint32) * 2 + 1  # odd, ascending, no equal neighbours
            if hit is not None and hit < length:
                j = 5 + hit
                if query in ("find_if", "count_if"):
                    x[j] = 6
                elif query == "adjacent_find" and j + 1 < 5 + length:
                    x[j + 1] = x[j]
                elif query == "is_sorted_until" and hit >= 1:
                    x[j] = x[j - 1] - 2
            op = {"find_if": "is_even", "count_if": "is_even", "adjacent_find": "equal",
                  "is_sorted_until": "less"}[query]
            np.testing.assert_array_equal(_run(ex, ex.to_device(x), off, query, op),
                                          orc.seg_query(x, off, query, op),
                                          err_msg=f"{length} {hit}")


def test_lazy_values(ex):
    from massively_b200 import lazy, op as O
    off = _lognormal_offsets(5000, 12)
    n = int(off[-1])
    x = seeded(np.int32, n, 2, hi=100)
    neg = (-x).astype(np.int32)
    got = _run(ex, lazy.map(ex.to_device(x), O.Negate), off, "find_if", "is_negative")
    np.testing.assert_array_equal(got, orc.seg_query(neg, off, "find_if", "is_negative"))
    got = _run(ex, lazy.counting(0).take(n), off, "is_sorted", "less")
    assert got.all()
