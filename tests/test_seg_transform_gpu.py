"""Per-segment transforms (Reverse, AdjacentDifference, Filter, Take,
Unique, Map): the CUDA path against the oracle (restating massively's
verification/oracle/src/seg.rs:41-153), exactly, on the reference's Take
test and on lognormal segmentations with empty and long segments, several
element types, and lazy values."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def _iter(ex, values, offsets_host):
    from massively_b200 import seg
    return seg.SegmentIterator(values, seg.Segmentation.from_offsets(ex, ex.to_device(offsets_host)))


def _offsets(nseg, seed):
    rng = np.random.default_rng(seed)
    lens = np.floor(rng.lognormal(1.5, 1.6, nseg) * 4).astype(np.int64)
    lens[rng.integers(0, nseg, max(1, nseg // 10))] = 0
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)


def test_take_known_answers(ex):
    from massively_b200 import seg
    for case in K.SEG_TAKE:
        r = seg.ForEachSegment(seg.Take(case["k"])).run(ex, _iter(ex, ex.to_device(case["x"]),
                                                                  case["offsets"]))
        np.testing.assert_array_equal(ex.to_host(r.values()), case["values"], err_msg=case["src"])
        np.testing.assert_array_equal(ex.to_host(r.offsets()), case["new_offsets"],
                                      err_msg=case["src"])


@pytest.mark.parametrize("nseg", [1, 9, 5000, 100_003])
@pytest.mark.parametrize("dtype", [np.uint8, np.int32, np.uint64, np.float32, np.float64])
def test_transforms(ex, nseg, dtype):
    from massively_b200 import op, seg
    off = _offsets(nseg, nseg + 1)
    n = int(off[-1])
    rng = np.random.default_rng(nseg)
    x = rng.integers(-3, 4, n).astype(dtype) if np.dtype(dtype).kind != "u" else \
        rng.integers(0, 4, n).astype(dtype)
    d = ex.to_device(x)
    cases = [(seg.Reverse(), "reverse", 0), (seg.AdjacentDifference(op.Max), "adjacent_difference",
                                             "max"),
             (seg.Unique(), "unique", 0), (seg.Take(3), "take", 3), (seg.Take(1000), "take", 1000),
             (seg.Filter(op.IsPositive), "filter", "is_positive")]
    if np.dtype(dtype).kind != "f":
        cases.append((seg.Filter(op.IsEven), "filter", "is_even"))
    for alg, kind, param in cases:
        r = seg.ForEachSegment(alg).run(ex, _iter(ex, d, off))
        wv, wo = orc.seg_transform(x, off, kind, param)
        np.testing.assert_array_equal(ex.to_host(r.values()), wv, err_msg=kind)
        np.testing.assert_array_equal(ex.to_host(r.offsets()), wo if kind in
                                      ("unique", "take", "filter") else off, err_msg=kind)


def test_long_segment_and_lazy_values(ex):
    from massively_b200 import lazy, op, seg
    off = np.array([0, 3, 3 + (1 << 20) + 7, (1 << 20) + 12], np.uint32)
    n = int(off[-1])
    r = seg.ForEachSegment(seg.Reverse()).run(ex, _iter(ex, lazy.counting(0).take(n), off))
    wv, _ = orc.seg_transform(np.arange(n, dtype=np.uint32), off, "reverse")
    np.testing.assert_array_equal(ex.to_host(r.values()), wv)
    r = seg.ForEachSegment(seg.Filter(op.IsOdd)).run(ex, _iter(ex, lazy.counting(0).take(n), off))
    wv, wo = orc.seg_transform(np.arange(n, dtype=np.uint32), off, "filter", "is_odd")
    np.testing.assert_array_equal(ex.to_host(r.values()), wv)
    np.testing.assert_array_equal(ex.to_host(r.offsets()), wo)
    m = seg.ForEachSegment(seg.Map(op.Negate)).run(
        ex, _iter(ex, ex.to_device(np.arange(n, dtype=np.int32)), off))
    np.testing.assert_array_equal(ex.to_host(m.values()), -np.arange(n, dtype=np.int32))
