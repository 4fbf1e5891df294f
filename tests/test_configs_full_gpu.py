"""The benchmark configurations at their full sizes, on their own seeded
inputs, against the oracle.

Each test builds the exact inputs the benchmark times (massively's PCG
streams at the configuration's seeds; normals by the host f64 Box-Muller of
bench.py; lognormal segment lengths and Zipf keys by bench.py's generators),
runs the CUDA path through the public API and compares every output with
the CPU oracle:

- integers, keys, indices, stability: bit-exact;
- f32 sums: against the FP64 oracle within n * 2^-24 * sum|x| per result
  (n = the number of terms: i + 1 for a prefix, the segment length for a
  segment), and bit-identical from run to run;
- f32 min / max: exact.

The sorted orders at 2^27 and 2^28 items come from oracle.radix_perm_par,
which gives the same permutation as the sequential oracle (a stable sort is
unique: it is the sort by (encoded key, input index)) on all host cores.
"""
import numpy as np
import pytest

import bench
from tests.gpu_util import executor, gpu

pytestmark = gpu

F32_EPS = 2.0 ** -24


@pytest.fixture(scope="module")
def ex():
    return executor()


def _free():
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _check_prefix_bound(got, x, what):
    """|got[i] - sum_{k<=i} x_k| <= (i+1) * 2^-24 * sum_{k<=i} |x_k|."""
    x64 = x.astype(np.float64)
    exact = np.cumsum(x64)
    bound = np.arange(1, x.size + 1, dtype=np.float64) * F32_EPS * np.cumsum(np.abs(x64))
    err = np.abs(got.astype(np.float64) - exact)
    bad = np.flatnonzero(err > bound)
    assert bad.size == 0, f"{what}: {bad.size} prefixes outside the bound, first at {bad[:5]}"


# ------------------------------------------------------------------- C1 --

def test_c1_plain_small_exact(ex, orc):
    """2^20 u32 keys uniform on [0, 2^32) from seed 0, values = index:
    inclusive_scan (wrapping add), reduce (add through a u64 view), and
    radix_sort_by_key(keys, zip2(keys, counting(0)))."""
    from massively_b200 import lazy, op, vector, zip2
    n = 1 << 20
    keys = orc.uniform_u32(0, 0xFFFFFFFF, 0, n)
    d = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 0, n)
    np.testing.assert_array_equal(ex.to_host(d), keys)  # the device stream is the oracle's
    scan = ex.to_host(vector.inclusive_scan(ex, d, op.Add))
    np.testing.assert_array_equal(scan, orc.inclusive_scan(keys, "add"))
    total = vector.reduce(ex, lazy.cast(d, np.uint64), np.uint64(0), op.Add)
    assert int(total) == int(orc.reduce(keys.astype(np.uint64), "add", 0))
    out = vector.radix_sort_by_key(ex, d, zip2(d, lazy.counting(0).take(n)))
    sk, sv = out.into_columns()
    perm = orc.radix_perm([keys])
    np.testing.assert_array_equal(ex.to_host(sv), perm)
    np.testing.assert_array_equal(ex.to_host(sk), keys[perm])


# ------------------------------------------------------------------- C2 --

@pytest.mark.parametrize("key_hi,seed", [(0xFFFFFFFF, 0), (65535, 1)])
def test_c2_sort_pairs_2e28_exact(ex, orc, key_hi, seed):
    """Stable sort_by_key of 2^28 (u32 key, u32 value = index) pairs, keys
    uniform 32-bit (seed 0) and uniform over 2^16 values (seed 1)."""
    from massively_b200 import lazy, vector
    n = 1 << 28
    kd = bench.device_uniform_u32(ex, 0, key_hi, seed, n)
    vd = ex.alloc(np.uint32, n)
    vector.copy(ex, lazy.counting(0).take(n), vd)
    sk, sv = vector.radix_sort_pairs(ex, kd, vd)
    keys = ex.to_host(kd)
    np.testing.assert_array_equal(keys[:4096], orc.uniform_u32(0, key_hi, seed, 4096))
    got_v, got_k = ex.to_host(sv), ex.to_host(sk)
    del kd, vd, sk, sv
    _free()
    perm = orc.radix_perm_par(keys)
    assert np.array_equal(got_v, perm), "values differ from the oracle's stable order"
    assert np.array_equal(got_k, keys[perm]), "keys differ from the oracle's stable order"


def test_c2_sort_u64_2e27_exact(ex, orc):
    """sort of 2^27 u64 keys uniform on the full range (seed 2), `<`."""
    from massively_b200 import op, vector
    n = 1 << 27
    kd = ex.alloc(np.uint64, n)
    from massively_b200 import _native as N
    from massively_b200.runtime import check
    check(N.lib().mb_random_uniform_u64(ex.handle, 0, 0xFFFFFFFFFFFFFFFF, 2, 0, kd.to_col()))
    got = ex.to_host(vector.sort(ex, kd, op.Less))
    keys = ex.to_host(kd)
    del kd
    _free()
    np.testing.assert_array_equal(keys[:4096], orc.uniform_u64(0, 0xFFFFFFFFFFFFFFFF, 2, 4096))
    assert np.array_equal(got, keys[orc.radix_perm_par(keys)])


def test_c2_scan_u32_2e30_exact(ex, orc):
    """inclusive_scan (wrapping add) of 2^30 u32 uniform (seed 3)."""
    from massively_b200 import op, vector
    n = 1 << 30
    xd = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 3, n)
    yd = vector.inclusive_scan(ex, xd, op.Add)
    x, y = ex.to_host(xd), ex.to_host(yd)
    del xd, yd
    _free()
    np.testing.assert_array_equal(x[:4096], orc.uniform_u32(0, 0xFFFFFFFF, 3, 4096))
    assert np.array_equal(y, orc.inclusive_scan(x, "add"))


def test_c2_scan_f32_2e28_bound_and_deterministic(ex):
    """inclusive_scan (add) of 2^28 f32 N(0,1) (seed 4): every prefix within
    the FP64 bound, and the same bits on a second run."""
    from massively_b200 import op, vector
    n = 1 << 28
    x = bench.host_normal_f32(ex, 4, n)
    xd = ex.to_device(x)
    y1 = ex.to_host(vector.inclusive_scan(ex, xd, op.Add))
    y2 = ex.to_host(vector.inclusive_scan(ex, xd, op.Add))
    del xd
    _free()
    assert np.array_equal(y1.view(np.uint32), y2.view(np.uint32)), "run-to-run bits differ"
    _check_prefix_bound(y1, x, "f32 scan 2^28")


def test_c2_copy_where_2e28_exact(ex, orc):
    """copy_where keeping k & 1 == 0 (a fused lazy predicate) of 2^28 u32
    (seed 5): the kept rows in order and their count."""
    from massively_b200 import lazy, op, vector
    n = 1 << 28
    xd = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 5, n)
    kept = vector.copy_where(ex, xd, lazy.map(xd, op.IsEven))
    cnt = kept.logical_len()
    got = ex.to_host(kept)[:cnt]
    x = ex.to_host(xd)
    del xd, kept
    _free()
    (want,) = orc.copy_where([x], ((x & 1) == 0).astype(np.uint32))
    assert cnt == want.size
    assert np.array_equal(got, want)


# ------------------------------------------------------------------- C3 --

@pytest.fixture(scope="module")
def c3(ex):
    """2^26 values in 2^20 segments with lognormal(3, 1.5) lengths (empty
    ones included), as the segmented benchmark builds them."""
    from massively_b200 import seg
    n, nseg = 1 << 26, 1 << 20
    off = bench.lognormal_offsets(ex, nseg, n, 106)
    assert off[-1] == n and (np.diff(off.astype(np.int64)) == 0).any()
    sgm = seg.Segmentation.from_offsets(ex, ex.to_device(off))
    return off, sgm


def test_c3_seg_scan_f32_bound(ex, orc, c3):
    from massively_b200 import op, seg
    off, sgm = c3
    x = bench.host_normal_f32(ex, 6, 1 << 26)
    xd = ex.to_device(x)
    it = sgm.segments(xd)
    y1 = ex.to_host(seg.ForEachSegment(seg.InclusiveScan(op.Add)).run(ex, it).values())
    y2 = ex.to_host(seg.ForEachSegment(seg.InclusiveScan(op.Add)).run(ex, it).values())
    assert np.array_equal(y1.view(np.uint32), y2.view(np.uint32)), "run-to-run bits differ"
    x64 = x.astype(np.float64)
    exact = orc.seg_inclusive_scan(x64, off, "add")
    absum = orc.seg_inclusive_scan(np.abs(x64), off, "add")
    lens = np.diff(off.astype(np.int64))
    local = np.arange(x.size, dtype=np.int64) - np.repeat(off[:-1].astype(np.int64), lens)
    bound = (local + 1) * F32_EPS * absum
    bad = np.flatnonzero(np.abs(y1.astype(np.float64) - exact) > bound)
    assert bad.size == 0, f"{bad.size} segment prefixes outside the bound, first at {bad[:5]}"


def test_c3_seg_reduce_f32(ex, orc, c3):
    """add within the per-segment bound; min and max exact; empty segments
    give init."""
    from massively_b200 import op, seg
    off, sgm = c3
    x = bench.host_normal_f32(ex, 6, 1 << 26)
    it = sgm.segments(ex.to_device(x))
    s = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Add, np.float32(0))).run(ex, it))
    lo = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Min, np.float32(np.inf))).run(ex, it))
    hi = ex.to_host(seg.ForEachSegment(seg.Reduce(op.Max, np.float32(-np.inf))).run(ex, it))
    x64 = x.astype(np.float64)
    exact = orc.seg_reduce(x64, off, "add", 0.0)
    absum = orc.seg_reduce(np.abs(x64), off, "add", 0.0)
    lens = np.diff(off.astype(np.int64))
    bad = np.flatnonzero(np.abs(s.astype(np.float64) - exact) > lens * F32_EPS * absum)
    assert bad.size == 0, f"{bad.size} segment sums outside the bound"
    np.testing.assert_array_equal(lo, orc.seg_reduce(x, off, "min", np.float32(np.inf)))
    np.testing.assert_array_equal(hi, orc.seg_reduce(x, off, "max", np.float32(-np.inf)))
    assert (s[lens == 0] == 0).all()


def test_c3_seg_sort_u32_exact(ex, orc, c3):
    """seg sort of u32 keys uniform per element (seed 6)."""
    from massively_b200 import op, seg
    off, sgm = c3
    kd = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 6, 1 << 26)
    got = ex.to_host(seg.ForEachSegment(seg.Sort(op.Less)).run(ex, sgm.segments(kd)).values())
    keys = ex.to_host(kd)
    assert np.array_equal(got, orc.seg_sort(keys, off, "less"))


# ------------------------------------------------------------------- C4 --

def test_c4_group_by_2e27_against_the_oracle_chain(ex, orc):
    """2^27 rows (u32 key Zipf(1.1) over 2^20 keys, f32 value N(0,1), u32
    flag Bernoulli(0.3)), as the captured graph runs them: copy_where on the
    flag -> sort_by_key -> reduce_by_key (f32 sum, u32 count, f32 min) ->
    set_intersection of the distinct keys with a sorted 2^20 u32 list.  The
    oracle runs the same chain step by step."""
    from massively_b200 import pipeline, vector
    n, nkeys, seed = 1 << 27, 1 << 20, 7
    keys_d = bench.zipf_keys(ex, n, nkeys, seed)
    _free()
    vals = bench.host_normal_f32(ex, seed + 1, n)
    vals_d = ex.to_device(vals)
    flag_d = bench.bernoulli_flags(ex, n, 0.3, seed + 2)
    other_d = vector.sort(ex, bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, seed + 3, 1 << 20))
    cap = pipeline.Captured(ex, lambda e: pipeline.group_by(e, keys_d, vals_d, flag_d, other_d))
    cap.replay()
    out = cap.outputs
    runs = out["keys"].logical_len()
    got = {k: ex.to_host(out[k])[:runs] for k in ("keys", "sum", "count", "min")}
    ncommon = out["common"].logical_len()
    got_common = ex.to_host(out["common"])[:ncommon]
    kept_n = out["kept"].logical_len()
    keys, flag, other = ex.to_host(keys_d), ex.to_host(flag_d), ex.to_host(other_d)
    del cap, out, keys_d, vals_d, flag_d, other_d
    _free()
    # the oracle chain
    k1, v1 = orc.copy_where([keys, vals], flag)
    assert kept_n == k1.size
    perm = orc.radix_perm_par(k1)
    sk, sv = k1[perm], v1[perm]
    heads = np.flatnonzero(np.concatenate([[True], sk[1:] != sk[:-1]]))
    np.testing.assert_array_equal(got["keys"], sk[heads])
    lens = np.diff(np.concatenate([heads, [sk.size]]))
    np.testing.assert_array_equal(got["count"], lens.astype(np.uint32))
    np.testing.assert_array_equal(got["min"], np.minimum.reduceat(sv, heads))
    sv64 = sv.astype(np.float64)
    exact = np.add.reduceat(sv64, heads)
    absum = np.add.reduceat(np.abs(sv64), heads)
    bad = np.flatnonzero(np.abs(got["sum"].astype(np.float64) - exact) > lens * F32_EPS * absum)
    assert bad.size == 0, f"{bad.size} run sums outside the bound"
    np.testing.assert_array_equal(got_common, orc.set_intersection(sk[heads], other))
