"""merge / merge_by_key and multiset set operations: CUDA path vs the
oracle, bit-exact (left-first ties, multiplicities)."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def test_known_answers(ex):
    from massively_b200 import op, vector
    for case in K.MERGE:
        got = vector.merge(ex, ex.to_device(case["left"]), ex.to_device(case["right"]), op.Less)
        np.testing.assert_array_equal(ex.to_host(got), case["want"])
    m = K.MERGE_BY_KEY
    got = vector.merge_by_key(ex, ex.to_device(m["lk"]), ex.to_device(m["lv"]),
                              ex.to_device(m["rk"]), ex.to_device(m["rv"]), op.Less)
    np.testing.assert_array_equal(ex.to_host(got), m["want"])
    for case in K.SETS:
        l, r = ex.to_device(case["left"]), ex.to_device(case["right"])
        np.testing.assert_array_equal(ex.to_host(vector.set_union(ex, l, r)), case["union"])
        np.testing.assert_array_equal(ex.to_host(vector.set_intersection(ex, l, r)),
                                      case["intersection"])
        np.testing.assert_array_equal(ex.to_host(vector.set_difference(ex, l, r)),
                                      case["difference"])


SIZES = [(0, 0), (0, 5), (7, 0), (1, 1), (31, 33), (255, 257), (1000, 3), (4096, 4096),
         (5000, 70_001), (1 << 20, 1 << 19)]


@pytest.mark.parametrize("nl,nr", SIZES)
@pytest.mark.parametrize("keyspace", [10, 1 << 20])
def test_merge_stable_with_payload(ex, nl, nr, keyspace):
    from massively_b200 import op, vector
    lk = np.sort(seeded(np.uint32, nl, 1) % np.uint32(keyspace)).astype(np.uint32)
    rk = np.sort(seeded(np.uint32, nr, 2) % np.uint32(keyspace)).astype(np.uint32)
    got = vector.merge(ex, ex.to_device(lk), ex.to_device(rk), op.Less)
    np.testing.assert_array_equal(ex.to_host(got), orc.merge(lk, rk))
    lv = np.arange(nl, dtype=np.uint32)
    rv = np.arange(nr, dtype=np.uint32) + np.uint32(1 << 30)
    got = vector.merge_by_key(ex, ex.to_device(lk), ex.to_device(lv), ex.to_device(rk),
                              ex.to_device(rv), op.Less)
    np.testing.assert_array_equal(ex.to_host(got), orc.merge_by_key(lk, lv, rk, rv)[1])


@pytest.mark.parametrize("dtype,less", [(np.int64, "greater"), (np.float32, "less"),
                                        (np.float64, "total_less")])
def test_merge_typed(ex, dtype, less):
    from massively_b200 import op, vector
    lk = orc.sort(seeded(dtype, 3000, 3), less)
    rk = orc.sort(seeded(dtype, 5000, 4), less)
    got = vector.merge(ex, ex.to_device(lk), ex.to_device(rk), op.pred2(less))
    np.testing.assert_array_equal(ex.to_host(got).view(np.uint8),
                                  orc.merge(lk, rk, less).view(np.uint8))


@pytest.mark.parametrize("nl,nr", SIZES)
@pytest.mark.parametrize("keyspace", [4, 1000, 1 << 30])
def test_set_ops_multiset(ex, nl, nr, keyspace):
    from massively_b200 import vector
    lk = np.sort(seeded(np.uint32, nl, 5) % np.uint32(keyspace)).astype(np.uint32)
    rk = np.sort(seeded(np.uint32, nr, 6) % np.uint32(keyspace)).astype(np.uint32)
    l, r = ex.to_device(lk), ex.to_device(rk)
    np.testing.assert_array_equal(ex.to_host(vector.set_union(ex, l, r)), orc.set_union(lk, rk))
    np.testing.assert_array_equal(ex.to_host(vector.set_intersection(ex, l, r)),
                                  orc.set_intersection(lk, rk))
    np.testing.assert_array_equal(ex.to_host(vector.set_difference(ex, l, r)),
                                  orc.set_difference(lk, rk))


@pytest.mark.parametrize("k,m", [(5000, 3000), (3000, 5000), (1, 7000), (7000, 0), (0, 9),
                                 (2304, 2304), (2305, 2303)])
def test_set_ops_take_copies_by_rank(ex, k, m):
    """Under LESS -0.0 and +0.0 are one value, so the bits show which input
    each output copy came from: intersection keeps the first min(k, m) left
    copies, difference the left copies past m, union every left copy and the
    right copies past k -- here in runs longer than a tile."""
    from massively_b200 import op, vector
    lo = np.sort(seeded(np.float32, 3000, 9)).astype(np.float32)
    hi = lo + np.float32(100.0)
    lk = np.concatenate([lo[lo < 0], np.full(k, -0.0, np.float32), hi]).astype(np.float32)
    rk = np.concatenate([lo[lo < 0][::2], np.full(m, 0.0, np.float32), hi[1::3]]).astype(
        np.float32)
    l, r = ex.to_device(lk), ex.to_device(rk)
    for name, fn in [("union", vector.set_union), ("intersection", vector.set_intersection),
                     ("difference", vector.set_difference)]:
        got = ex.to_host(fn(ex, l, r, op.Less))
        want = getattr(orc, f"set_{name}")(lk, rk, "less")
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=name)


@pytest.mark.parametrize("dtype,less", [(np.int64, "greater"), (np.float64, "total_less"),
                                        (np.uint8, "less"), (np.int16, "less")])
def test_set_ops_typed(ex, dtype, less):
    from massively_b200 import op, vector
    lk = orc.sort(seeded(dtype, 20_000, 13, lo=0, hi=50) if np.dtype(dtype).kind in "iu"
                  else seeded(dtype, 20_000, 13), less)
    rk = orc.sort(seeded(dtype, 9_000, 14, lo=0, hi=50) if np.dtype(dtype).kind in "iu"
                  else seeded(dtype, 9_000, 14), less)
    if np.dtype(dtype).kind == "f":
        rk = orc.sort(np.concatenate([rk, lk[::7]]).astype(dtype), less)
    l, r = ex.to_device(lk), ex.to_device(rk)
    p = op.pred2(less)
    for name, fn in [("union", vector.set_union), ("intersection", vector.set_intersection),
                     ("difference", vector.set_difference)]:
        got = ex.to_host(fn(ex, l, r, p))
        want = getattr(orc, f"set_{name}")(lk, rk, less)
        np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8), err_msg=name)


def test_set_ops_device_length_and_lazy_inputs(ex):
    """Inputs whose logical lengths are device counts (a copy_where result)
    and lazy views (counting, map)."""
    from massively_b200 import lazy, op, vector
    n = 50_000
    x = np.sort(seeded(np.uint32, n, 15) % np.uint32(5000)).astype(np.uint32)
    st = (seeded(np.uint32, n, 16) % 3 != 0).astype(np.uint32)
    kept = vector.copy_where(ex, ex.to_device(x), ex.to_device(st))
    xk = x[st != 0]
    cnt = lazy.counting(100).take(3000)  # 100 .. 3099
    c_host = np.arange(100, 3100, dtype=np.uint32)
    for name, fn in [("union", vector.set_union), ("intersection", vector.set_intersection),
                     ("difference", vector.set_difference)]:
        got = fn(ex, kept, cnt)
        h = ex.to_host(got)[:got.logical_len()] if got.len_dev is not None else ex.to_host(got)
        np.testing.assert_array_equal(h, getattr(orc, f"set_{name}")(xk, c_host), err_msg=name)
        got = fn(ex, cnt, kept)
        h = ex.to_host(got)[:got.logical_len()] if got.len_dev is not None else ex.to_host(got)
        np.testing.assert_array_equal(h, getattr(orc, f"set_{name}")(c_host, xk), err_msg=name)
    # all inputs empty at run time
    none = vector.copy_where(ex, ex.to_device(x[:10]), ex.to_device(np.zeros(10, np.uint32)))
    got = vector.set_union(ex, none, none)
    assert got.logical_len() == 0
