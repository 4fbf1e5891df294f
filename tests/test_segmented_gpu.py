"""Segmented scan / reduce / sort over a Segmentation, and the by-key
algorithms: CUDA path vs the oracle (bit-exact for integers, FP64-oracle
bounds for f32)."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def _lognormal_offsets(nseg, total, seed):
    """Segment lengths lognormal(mu=3, sigma=1.5) rescaled to sum to `total`
    (largest remainder), empty segments allowed -- the segmented workload's
    shape at test size."""
    rng = np.random.default_rng(seed)
    raw = rng.lognormal(3.0, 1.5, nseg)
    scaled = raw / raw.sum() * total
    base = np.floor(scaled).astype(np.int64)
    rem = total - int(base.sum())
    order = np.argsort(-(scaled - base), kind="stable")
    base[order[:rem]] += 1
    return np.concatenate([[0], np.cumsum(base)]).astype(np.uint32)


def _strategy_offsets(seed):
    """massively's seg oracle strategy: 0-5 segments, lengths from
    SEGMENT_LENGTHS (verification/oracle/tests/seg.rs:20-28)."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(0, 6))
    lens = rng.choice(K.SEGMENT_LENGTHS, size=k)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)


def test_known_answers(ex):
    from massively_b200 import op, seg
    for case in K.SEG:
        s = seg.Segmentation.from_offsets(ex, ex.to_device(case["offsets"]))
        it = s.segments(ex.to_device(case["x"]))
        if case["kind"] == "reduce":
            got = seg.ForEachSegment(seg.Reduce(op.Add, np.uint32(case["init"]))).run(ex, it)
            np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
        else:
            got = seg.ForEachSegment(seg.ExclusiveScan(op.Add, np.uint32(case["init"]))).run(ex, it)
            np.testing.assert_array_equal(ex.to_host(got.values()), case["want"])


def test_segmentation_constructors(ex):
    import massively_b200 as mb
    from massively_b200 import lazy, seg
    for case in K.SEGMENTATION:
        s = seg.Segmentation.from_lengths(ex, ex.to_device(case["lengths"]))
        np.testing.assert_array_equal(ex.to_host(s.offsets()), case["offsets"])
        assert s.segment_count() == case["lengths"].size
        assert s.value_count() == int(case["offsets"][-1])
        np.testing.assert_array_equal(ex.to_host(s.segment_ids(ex)), case["ids"])
        np.testing.assert_array_equal(ex.to_host(s.local_indices(ex)), case["local"])
        s2 = seg.Segmentation.from_offsets(ex, ex.to_device(case["offsets"]))
        np.testing.assert_array_equal(ex.to_host(s2.lengths(ex)), case["lengths"])
        s3 = seg.Segmentation.from_segment_ids(ex, ex.to_device(case["ids"]),
                                               case["lengths"].size)
        np.testing.assert_array_equal(ex.to_host(s3.offsets()), case["offsets"])
    s = seg.Segmentation.from_lengths(ex, lazy.constant(np.uint32(2)).take(3))
    np.testing.assert_array_equal(ex.to_host(s.offsets()), [0, 2, 4, 6])
    for bad in K.INVALID_OFFSETS["cases"]:
        with pytest.raises(mb.InvalidSegmentation):
            seg.Segmentation.from_offsets(ex, ex.to_device(bad))
    with pytest.raises(mb.LengthTooLarge):
        seg.Segmentation.from_lengths(ex, ex.to_device(K.OVERFLOWING_LENGTHS["lengths"]))
    for ids in ([0, 2, 1], [0, 3]):
        with pytest.raises(mb.InvalidSegmentation):
            seg.Segmentation.from_segment_ids(ex, ex.to_device(np.array(ids, np.uint32)), 3)


def _run_all(ex, x, off, dtype):
    from massively_b200 import op, seg
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    it = s.segments(ex.to_device(x))
    out = {}
    out["incl"] = ex.to_host(seg.ForEachSegment(seg.InclusiveScan(op.Add)).run(ex, it).values())
    out["excl"] = ex.to_host(seg.ForEachSegment(seg.ExclusiveScan(op.Add, dtype(3))).run(ex, it)
                             .values())
    for name, o, init in (("add", op.Add, dtype(3)), ("min", op.Min, dtype(100)),
                          ("max", op.Max, dtype(0))):
        out["red_" + name] = ex.to_host(seg.ForEachSegment(seg.Reduce(o, init)).run(ex, it))
    out["sort"] = ex.to_host(seg.ForEachSegment(seg.Sort(op.Less)).run(ex, it).values())
    return out


@pytest.mark.parametrize("seed", range(24))
def test_oracle_strategy_u32(ex, seed):
    off = _strategy_offsets(seed)
    n = int(off[-1])
    x = (seeded(np.uint32, n, seed) % 100).astype(np.uint32)
    got = _run_all(ex, x, off, np.uint32)
    np.testing.assert_array_equal(got["incl"], orc.seg_inclusive_scan(x, off, "add"))
    np.testing.assert_array_equal(got["excl"], orc.seg_exclusive_scan(x, off, "add", 3))
    np.testing.assert_array_equal(got["red_add"], orc.seg_reduce(x, off, "add", 3))
    np.testing.assert_array_equal(got["red_min"], orc.seg_reduce(x, off, "min", 100))
    np.testing.assert_array_equal(got["red_max"], orc.seg_reduce(x, off, "max", 0))
    np.testing.assert_array_equal(got["sort"], orc.seg_sort(x, off, "less"))


@pytest.mark.parametrize("nseg,total", [(7, 4096), (100, 4097), (1 << 12, 1 << 18),
                                        (1 << 16, 1 << 22), (1 << 20, 1 << 23)])
def test_lognormal_u32_bit_exact(ex, nseg, total):
    off = _lognormal_offsets(nseg, total, nseg)
    x = seeded(np.uint32, total, 5)
    got = _run_all(ex, x, off, np.uint32)
    np.testing.assert_array_equal(got["incl"], orc.seg_inclusive_scan(x, off, "add"))
    np.testing.assert_array_equal(got["excl"], orc.seg_exclusive_scan(x, off, "add", 3))
    np.testing.assert_array_equal(got["red_add"], orc.seg_reduce(x, off, "add", 3))
    np.testing.assert_array_equal(got["red_min"], orc.seg_reduce(x, off, "min", 100))
    np.testing.assert_array_equal(got["red_max"], orc.seg_reduce(x, off, "max", 0))
    np.testing.assert_array_equal(got["sort"], orc.seg_sort(x, off, "less"))


@pytest.mark.parametrize("nseg,total", [(100, 4097), (1 << 16, 1 << 22)])
def test_lognormal_f32_against_fp64(ex, nseg, total):
    from massively_b200 import op, seg
    off = _lognormal_offsets(nseg, total, 3)
    x = orc.normal_f32(7, total)
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    it = s.segments(ex.to_device(x))
    incl = ex.to_host(seg.ForEachSegment(seg.InclusiveScan(op.Add)).run(ex, it).values())
    red = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Add, np.float32(0))).run(ex, it))
    x64 = x.astype(np.float64)
    want_incl = orc.seg_inclusive_scan(x64, off, "add")
    want_red = orc.seg_reduce(x64, off, "add", 0.0)
    lens = np.diff(off.astype(np.int64))
    abs_sum = orc.seg_reduce(np.abs(x64), off, "add", 0.0)
    # per segment: |err| <= len * 2^-24 * sum|x|
    assert (np.abs(red - want_red) <= lens * 2.0 ** -24 * abs_sum + 1e-30).all()
    abs_pref = orc.seg_inclusive_scan(np.abs(x64), off, "add")
    local = np.arange(total) - np.repeat(off[:-1].astype(np.int64), lens)
    assert (np.abs(incl - want_incl) <= (local + 1) * 2.0 ** -24 * abs_pref + 1e-30).all()
    # min / max are exact
    mn = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Min, np.float32(np.inf))).run(ex, it))
    np.testing.assert_array_equal(mn, orc.seg_reduce(x, off, "min", np.float32(np.inf)))
    mx = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Max, np.float32(-np.inf))).run(ex, it))
    np.testing.assert_array_equal(mx, orc.seg_reduce(x, off, "max", np.float32(-np.inf)))
    # deterministic
    red2 = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Add, np.float32(0))).run(ex, it))
    np.testing.assert_array_equal(red.view(np.uint32), red2.view(np.uint32))


def test_all_empty_and_trailing_empty_segments(ex):
    from massively_b200 import op, seg
    off = np.array([0, 0, 0, 5, 5, 9, 9, 9], np.uint32)
    x = np.arange(9, dtype=np.uint32)
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    got = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Add, np.uint32(7))).run(ex, s.segments(
        ex.to_device(x))))
    np.testing.assert_array_equal(got, orc.seg_reduce(x, off, "add", 7))
    off = np.array([0, 0, 0], np.uint32)
    s = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    got = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Add, np.uint32(7))).run(
        ex, s.segments(ex.to_device(np.zeros(0, np.uint32)))))
    np.testing.assert_array_equal(got, [7, 7])


# ------------------------------------------------------------------ by key --

def test_by_key_known_answers(ex):
    from massively_b200 import op, vector, zip7
    for case in K.BY_KEY:
        k, v = ex.to_device(case["keys"]), ex.to_device(case["values"])
        if case["kind"] == "reduce":
            ok, ov = vector.reduce_by_key(ex, k, v, op.Equal, np.uint32(case["init"]), op.Add)
            np.testing.assert_array_equal(ex.to_host(ok), case["want_keys"])
            np.testing.assert_array_equal(ex.to_host(ov), case["want"])
        elif case["kind"] == "inclusive":
            got = vector.inclusive_scan_by_key(ex, k, v, op.Equal, op.Add)
            np.testing.assert_array_equal(ex.to_host(got), case["want"])
        else:
            got = vector.exclusive_scan_by_key(ex, k, v, op.Equal, np.uint32(case["init"]),
                                               op.Add)
            np.testing.assert_array_equal(ex.to_host(got), case["want"])
    s = K.BY_KEY_SEVEN
    n = s["n"]
    keys = ex.to_device(np.where(np.arange(n) < 300, 1, 2).astype(np.uint32))
    cols = zip7(*[ex.to_device(np.full(n, c, np.uint32)) for c in range(1, 8)])
    inc = vector.inclusive_scan_by_key(ex, keys, cols, op.Equal, op.Add).into_columns()
    a, g = ex.to_host(inc[0]), ex.to_host(inc[6])
    assert (a[299], a[300], a[599]) == (300, 1, 300)
    assert (g[299], g[300], g[599]) == (2100, 7, 2100)
    inits = tuple(np.uint32(i) for i in s["inits"])
    exc = vector.exclusive_scan_by_key(ex, keys, cols, op.Equal, inits, op.Add).into_columns()
    e = ex.to_host(exc[0])
    assert (e[0], e[1], e[300], e[301]) == (10, 11, 10, 11)
    ok, ov = vector.reduce_by_key(ex, keys, cols, op.Equal, inits, op.Add)
    np.testing.assert_array_equal(ex.to_host(ok), [1, 2])
    np.testing.assert_array_equal(ex.to_host(ov.into_columns()[0]), [310, 310])
    np.testing.assert_array_equal(ex.to_host(ov.into_columns()[6]), [2170, 2170])


@pytest.mark.parametrize("n", K.ORACLE_LENGTHS + [4097, 65_537, 1 << 20])
def test_reduce_by_key_strategy(ex, n):
    # massively's by-key strategy: keys from 0..12, values 0..50
    # (verification/oracle/tests/vector/by_key.rs:12), sorted keys here so
    # runs are long, plus an unsorted variant (short runs).
    from massively_b200 import op, vector
    for sort_keys in (True, False):
        keys = (seeded(np.uint32, n, n) % 12).astype(np.uint32)
        if sort_keys:
            keys = np.sort(keys)
        vals = (seeded(np.uint32, n, n + 1) % 50).astype(np.uint32)
        ok, ov = vector.reduce_by_key(ex, ex.to_device(keys), ex.to_device(vals), op.Equal,
                                      np.uint32(0), op.Add)
        wk, wv = orc.reduce_by_key(keys, vals, "add", 0)
        np.testing.assert_array_equal(ex.to_host(ok), wk)
        np.testing.assert_array_equal(ex.to_host(ov), wv)
        got = vector.inclusive_scan_by_key(ex, ex.to_device(keys), ex.to_device(vals), op.Equal,
                                           op.Add)
        np.testing.assert_array_equal(ex.to_host(got), orc.scan_by_key(keys, vals, "add"))
        got = vector.exclusive_scan_by_key(ex, ex.to_device(keys), ex.to_device(vals), op.Equal,
                                           np.uint32(4), op.Max)
        np.testing.assert_array_equal(ex.to_host(got),
                                      orc.scan_by_key(keys, vals, "max", True, 4))


def test_group_by_columns(ex):
    # the group-by shape: (sum f32, count u32 via constant(1), min f32) per key
    from massively_b200 import lazy, op, vector, zip3
    n = 1 << 20
    keys = np.sort((seeded(np.uint32, n, 1) % 5000).astype(np.uint32))
    vals = orc.normal_f32(2, n)
    dk, dv = ex.to_device(keys), ex.to_device(vals)
    ok, ov = vector.reduce_by_key(
        ex, dk, zip3(dv, lazy.constant(np.uint32(1)).take(n), dv), op.Equal,
        (np.float32(0), np.uint32(0), np.float32(np.inf)), (op.Add, op.Add, op.Min))
    s, c, m = ov.into_columns()
    wk, (ws, wc, wm) = orc.reduce_by_key(keys, [vals.astype(np.float64), np.ones(n, np.uint32),
                                                vals], ["add", "add", "min"],
                                         [0.0, 0, np.float32(np.inf)])
    np.testing.assert_array_equal(ex.to_host(ok), wk)
    np.testing.assert_array_equal(ex.to_host(c), wc)
    np.testing.assert_array_equal(ex.to_host(m), wm)
    abs_sum = orc.reduce_by_key(keys, np.abs(vals.astype(np.float64)), "add", 0.0)[1]
    assert (np.abs(ex.to_host(s) - ws) <= wc * 2.0 ** -24 * abs_sum + 1e-30).all()


@pytest.mark.parametrize("n", [1, 4095, 4097, 70_001, 1 << 20])
def test_constant_columns_count_runs(ex, n):
    # Constant integer columns under ADD come from the run lengths (no value
    # pass): first in the zip (another column writes the keys), 64-bit, signed
    # with a negative constant, beside a plain column and a non-ADD constant;
    # and the segmented form, whose runs also break at segment starts.
    from massively_b200 import lazy, op, vector, zip4
    keys = np.sort((seeded(np.uint32, n, 7) % max(1, n // 37)).astype(np.uint32))
    vals = (seeded(np.uint32, n, 8) % 1000).astype(np.uint32)
    dk, dv = ex.to_device(keys), ex.to_device(vals)
    cols = zip4(lazy.constant(np.uint32(3)).take(n), dv, lazy.constant(np.int64(-2)).take(n),
                lazy.constant(np.uint32(5)).take(n))
    inits = (np.uint32(7), np.uint32(0), np.int64(11), np.uint32(9))
    ops = (op.Add, op.Add, op.Add, op.Max)
    ok, ov = vector.reduce_by_key(ex, dk, cols, op.Equal, inits, ops)
    a, b, c, d = (ex.to_host(x) for x in ov.into_columns())
    wk, (wa, wb, wc, wd) = orc.reduce_by_key(
        keys, [np.full(n, 3, np.uint32), vals, np.full(n, -2, np.int64), np.full(n, 5, np.uint32)],
        ["add", "add", "add", "max"], [7, 0, 11, 9])
    np.testing.assert_array_equal(ex.to_host(ok), wk)
    for got, want in ((a, wa), (b, wb), (c, wc), (d, wd)):
        np.testing.assert_array_equal(got, want)
    # segmented: segment starts every 1000 items also end runs
    off = np.arange(0, n + 1000, 1000, dtype=np.uint32)
    off[-1] = n
    off = np.unique(np.minimum(off, n)).astype(np.uint32)
    sk, sv = vector.reduce_by_key_segmented(ex, dk, cols, op.Equal, inits, ops, ex.to_device(off))
    heads = np.ones(n, bool)
    heads[1:] = keys[1:] != keys[:-1]
    heads[off[:-1]] = True
    starts = np.flatnonzero(heads)
    lens = np.diff(np.append(starts, n)).astype(np.uint64)
    np.testing.assert_array_equal(ex.to_host(sk), keys[starts])
    sa, sb, sc, sd = (ex.to_host(x) for x in sv.into_columns())
    np.testing.assert_array_equal(sa, (7 + 3 * lens).astype(np.uint32))
    np.testing.assert_array_equal(sc, (11 - 2 * lens.astype(np.int64)).astype(np.int64))
    np.testing.assert_array_equal(sb, np.add.reduceat(vals.astype(np.uint64), starts).astype(np.uint32))
    np.testing.assert_array_equal(sd, np.full(starts.size, 9, np.uint32))
