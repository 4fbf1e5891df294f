"""ForEachSegment(Sort): the shared-memory segmented sort of 4-byte values
(packs of short segments per range, long segments one per CTA, the global
radix path past the one-CTA limit) against the oracle's per-segment stable
sort (verification/oracle/src/seg.rs:18-39), bit-exact."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu

RANGE = 2048      # start positions per range (csrc/segsort.cu kSsRange)
TILE = 4096       # one CTA's shared-memory tile (kSsTile)
LONG_LIMIT = 1 << 17  # longest segment one CTA sorts (kSsLongLimit)


@pytest.fixture(scope="module")
def ex():
    return executor()


def _offsets(lengths):
    return np.concatenate([[0], np.cumsum(np.asarray(lengths, np.int64))]).astype(np.uint32)


def _run(ex, x, off, less, view=None):
    from massively_b200 import op, seg
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    vals = ex.to_device(x) if view is None else view(ex.to_device(x))
    pred = {"less": op.Less, "greater": op.Greater, "total_less": op.TotalLess}[less]
    return ex.to_host(seg.ForEachSegment(seg.Sort(pred)).run(ex, s.segments(vals)).values())


def _values(dtype, n, seed):
    u = seeded(np.uint32, n, seed)
    if dtype == np.float32:
        # Finite floats over many binades, with signed zeros mixed in.
        f = ((u >> 9).astype(np.float32) / np.float32(1 << 23) - np.float32(0.5)) * \
            np.exp2(((u & 0xFF).astype(np.int32) % 40) - 20).astype(np.float32)
        f[u % 17 == 0] = np.float32(0.0)
        f[u % 19 == 0] = np.float32(-0.0)
        return f.astype(np.float32)
    return u.view(dtype)


# Every size class: empty, one item, short packs, a segment just under and
# just over the range, over a tile (one CTA per segment), and starts on range
# edges.
CLASS_LENGTHS = [0, 1, 2, 31, 32, 33, 0, 2047, 2048, 2049, 1, 4095, 4096, 4097, 3, 0, 0,
                 RANGE * 3, 8191, 10_000, 5, 65_000, 7, LONG_LIMIT, 2, 0]


@pytest.mark.parametrize("dtype", [np.uint32, np.int32, np.float32])
@pytest.mark.parametrize("less", ["less", "greater", "total_less"])
def test_size_classes(ex, dtype, less):
    off = _offsets(CLASS_LENGTHS)
    x = _values(dtype, int(off[-1]), 11)
    got = _run(ex, x, off, less)
    want = orc.seg_sort(x, off, less)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("dtype", [np.uint32, np.float32])
@pytest.mark.parametrize("nseg,total", [(1, 5000), (3, 3 * RANGE), (2000, 4000),
                                        (1 << 14, 1 << 20), (1 << 20, 1 << 23)])
def test_lognormal_and_dense(ex, dtype, nseg, total):
    rng = np.random.default_rng(nseg)
    raw = rng.lognormal(3.0, 1.5, nseg)
    lens = np.floor(raw / raw.sum() * total).astype(np.int64)
    lens[0] += total - lens.sum()
    off = _offsets(lens)
    x = _values(dtype, total, nseg)
    for less in ("less", "total_less"):
        got = _run(ex, x, off, less)
        assert np.array_equal(got.view(np.uint32), orc.seg_sort(x, off, less).view(np.uint32))


def test_many_segments_in_one_pack(ex):
    # Ranges holding hundreds of tiny segments: the segment index inside a
    # pack takes more than 8 bits (two index passes).
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 4, 30_000)
    off = _offsets(lens)
    x = seeded(np.uint32, int(off[-1]), 4)
    assert np.array_equal(_run(ex, x, off, "less"), orc.seg_sort(x, off, "less"))


def test_empty_segment_runs(ex):
    # 10^4 empty segments in one place, empties at both ends, all-empty.
    lens = [0] * 5 + [40] + [0] * 10_000 + [3000, 1] + [0] * 7
    off = _offsets(lens)
    x = seeded(np.uint32, int(off[-1]), 5)
    assert np.array_equal(_run(ex, x, off, "less"), orc.seg_sort(x, off, "less"))
    off = _offsets([0] * 9)
    assert _run(ex, np.zeros(0, np.uint32), off, "less").size == 0


def test_constant_digits_and_equal_keys(ex):
    # Values below 256 (three constant digits skipped) and all-equal
    # segments, including a long one (no pass at all).
    lens = [100, 5000, 3000, 20_000, 17]
    off = _offsets(lens)
    n = int(off[-1])
    x = (seeded(np.uint32, n, 6) % 200).astype(np.uint32)
    x[100:5100] = 7
    x[8100:28100] = 9
    assert np.array_equal(_run(ex, x, off, "less"), orc.seg_sort(x, off, "less"))
    assert np.array_equal(_run(ex, x, off, "greater"), orc.seg_sort(x, off, "greater"))


def test_signed_zeros_keep_input_order(ex):
    # Under `<` -0.0 and +0.0 tie: the sort is stable, so their bits come out
    # in input order, in short and long segments alike.
    n1, n2 = 300, 20_000
    x = np.where(seeded(np.uint32, n1 + n2, 7) % 2 == 0, np.float32(0.0), np.float32(-0.0))
    x = x.astype(np.float32)
    x[::5] = np.float32(1.5)
    off = _offsets([n1, n2])
    for less in ("less", "greater"):
        got = _run(ex, x, off, less)
        assert np.array_equal(got.view(np.uint32), orc.seg_sort(x, off, less).view(np.uint32))


def test_total_order_specials(ex):
    vals = np.array([np.nan, -np.inf, np.inf, -0.0, 0.0, 1e-45, -1e-45, 3.0e38, -np.nan],
                    np.float32)
    x = np.tile(vals, 800)
    off = _offsets([9, 90, 900, 6201])
    got = _run(ex, x, off, "total_less")
    assert np.array_equal(got.view(np.uint32), orc.seg_sort(x, off, "total_less").view(np.uint32))


def test_past_the_one_cta_limit(ex):
    # A segment longer than one CTA sorts takes the global radix path; the
    # results are the same.
    lens = [10, LONG_LIMIT + 1, 4000, 3]
    off = _offsets(lens)
    x = seeded(np.int32, int(off[-1]), 8)
    assert np.array_equal(_run(ex, x, off, "less"), orc.seg_sort(x, off, "less"))
    lens = [300_000]
    off = _offsets(lens)
    x = seeded(np.uint32, 300_000, 9)
    assert np.array_equal(_run(ex, x, off, "less"), orc.seg_sort(x, off, "less"))


def test_lazy_values(ex):
    from massively_b200 import lazy
    lens = [5, 3000, 9000, 1, 40]
    off = _offsets(lens)
    x = seeded(np.uint32, int(off[-1]), 10)
    got = _run(ex, x, off, "less", view=lambda d: lazy.reverse(d))
    assert np.array_equal(got, orc.seg_sort(x[::-1].copy(), off, "less"))


def test_graph_capture_replays(ex):
    # Inside a capture the host cannot read the classification, so every
    # segment longer than a tile goes to the long-segment CTAs.
    import torch
    from massively_b200 import op, pipeline, seg
    lens = [1000, 9000, 3, 70_000, 2500]
    off = _offsets(lens)
    x = seeded(np.uint32, int(off[-1]), 12)
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    xd = ex.to_device(x)
    cap = pipeline.Captured(ex, lambda e: seg.ForEachSegment(seg.Sort(op.Less)).run(
        e, s.segments(xd)).values())
    want = orc.seg_sort(x, off, "less")
    for _ in range(2):
        cap.replay()
        torch.cuda.synchronize()
        assert np.array_equal(ex.to_host(cap.outputs), want)
    cap.release()


@pytest.mark.parametrize("less", ["less", "greater"])
def test_runs_equal_in_the_high_digits(ex, less):
    # The passes leave out the lowest varying digits and order the runs of
    # keys that agree on the rest afterwards: short runs out of order, long
    # runs already in order (duplicates), and long runs out of order (the
    # whole pack sorted again with every digit).
    n = 40_000
    u = seeded(np.uint32, n, 13)
    lens = [1500, 2000, 300, 4000, 20_000, 2100, 10_100]
    off = _offsets(lens)
    # every digit varies, the top three from one bit each, the lowest is
    # random: keys agree on the top three digits in long runs
    x = ((u >> 31) << 24) | (((u >> 30) & 1) << 16) | (((u >> 29) & 1) << 8) | (u & 0xFF)
    x = x.astype(np.uint32)
    # a stretch of one repeated value (a long run in order)
    x[1500:3000] = 0x12345678
    # a stretch of full-range values (runs of two or three, rarely)
    x[3500:3800] = seeded(np.uint32, 300, 14)
    x[30_000:40_000] = seeded(np.uint32, 10_000, 15)
    got = _run(ex, x, off, less)
    assert np.array_equal(got, orc.seg_sort(x, off, less))
    f = (x.view(np.float32) * np.float32(1)).astype(np.float32)
    f[np.isnan(f)] = np.float32(-0.0)
    got = _run(ex, f, off, less)
    assert np.array_equal(got.view(np.uint32), orc.seg_sort(f, off, less).view(np.uint32))
