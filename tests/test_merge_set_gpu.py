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
