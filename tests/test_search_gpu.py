"""lower_bound / upper_bound: the CUDA path against the oracle (restating
massively's verification/oracle/src/vector.rs:404-426), bit-exact, on the
reference's doctest and on seeded inputs across sizes, duplicates, values
beyond both ends, empty inputs, types and predicates."""
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
    from massively_b200 import vector
    for case in K.BOUNDS:
        src, vals = ex.to_device(case["source"]), ex.to_device(case["values"])
        np.testing.assert_array_equal(ex.to_host(vector.lower_bound(ex, src, vals)), case["lower"])
        np.testing.assert_array_equal(ex.to_host(vector.upper_bound(ex, src, vals)), case["upper"])


@pytest.mark.parametrize("n", [0, 1, 7, 4095, 4096, 4097, 100_003, 1 << 20])
@pytest.mark.parametrize("m", [0, 1, 1000, 70_001])
@pytest.mark.parametrize("span", [16, 1 << 30])
def test_u32_bounds(ex, n, m, span):
    from massively_b200 import vector
    src = np.sort(seeded(np.uint32, n, n + 3, hi=span - 1)) if n else np.empty(0, np.uint32)
    vals = seeded(np.uint32, m, m + 11, hi=span + 5)
    ds, dv = ex.to_device(src), ex.to_device(vals)
    np.testing.assert_array_equal(ex.to_host(vector.lower_bound(ex, ds, dv)),
                                  orc.lower_bound(src, vals))
    np.testing.assert_array_equal(ex.to_host(vector.upper_bound(ex, ds, dv)),
                                  orc.upper_bound(src, vals))


@pytest.mark.parametrize("dtype", [np.int32, np.float32, np.uint64, np.int64, np.float64,
                                   np.uint8, np.int16])
@pytest.mark.parametrize("less", ["less", "greater", "total_less"])
def test_types_and_predicates(ex, dtype, less):
    from massively_b200 import op, vector
    rng = np.random.default_rng(5)
    n, m = 50_000, 20_000
    if np.dtype(dtype).kind == "f":
        src = rng.normal(size=n).astype(dtype)
        vals = rng.normal(size=m).astype(dtype)
        vals[:10] = src[:10]  # exact hits
    else:
        info = np.iinfo(dtype)
        src = rng.integers(max(info.min, -1000), min(info.max, 1000), n).astype(dtype)
        vals = rng.integers(max(info.min, -1100), min(info.max, 1100), m).astype(dtype)
    order = orc.sort_perm(src, less)
    src = src[order]
    pred = {"less": op.Less, "greater": op.Greater, "total_less": op.TotalLess}[less]
    ds, dv = ex.to_device(src), ex.to_device(vals)
    np.testing.assert_array_equal(ex.to_host(vector.lower_bound(ex, ds, dv, pred)),
                                  orc.lower_bound(src, vals, less))
    np.testing.assert_array_equal(ex.to_host(vector.upper_bound(ex, ds, dv, pred)),
                                  orc.upper_bound(src, vals, less))


def test_lazy_values_and_errors(ex):
    import massively_b200 as mb
    from massively_b200 import lazy, vector
    src = np.arange(0, 2000, 2, dtype=np.uint32)
    ds = ex.to_device(src)
    got = vector.lower_bound(ex, ds, lazy.counting(0).take(2001))
    np.testing.assert_array_equal(ex.to_host(got), orc.lower_bound(src, np.arange(2001,
                                                                                  dtype=np.uint32)))
    with pytest.raises(mb.Launch):
        vector.lower_bound(ex, ds, ex.to_device(np.zeros(3, np.float32)))


def test_unique_known_answers(ex):
    from massively_b200 import vector
    for case in K.UNIQUE:
        got = vector.unique(ex, ex.to_device(case["x"]))
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    # by_key.rs doctest of unique_by_key
    k = ex.to_device(np.array([1, 1, 2, 2, 3], np.uint32))
    v = ex.to_device(np.array([10, 11, 20, 21, 30], np.uint32))
    np.testing.assert_array_equal(ex.to_host(vector.unique_by_key(ex, k, v)), [10, 20, 30])


@pytest.mark.parametrize("n", [0, 1, 2, 8191, 8192, 8193, 300_001])
@pytest.mark.parametrize("dtype", [np.uint32, np.int64, np.float32, np.uint16])
def test_unique_and_by_key(ex, n, dtype):
    from massively_b200 import iter as I, vector
    rng = np.random.default_rng(n + 1)
    x = np.sort(rng.integers(0, max(1, n // 3), n)).astype(dtype)
    if np.dtype(dtype).kind == "f" and n > 4:
        x[1] = np.nan
        x[2] = np.nan
        x[3] = -0.0
        x[4] = 0.0
    np.testing.assert_array_equal(ex.to_host(vector.unique(ex, ex.to_device(x))), orc.unique(x))
    heads = np.concatenate([[True], x[1:] != x[:-1]]) if n else np.zeros(0, bool)
    vals = np.arange(n, dtype=np.uint32)
    got = vector.unique_by_key(ex, ex.to_device(x), I.Zip(ex.to_device(vals), ex.to_device(x)))
    a, b = got.cols
    np.testing.assert_array_equal(ex.to_host(a), vals[heads])
    np.testing.assert_array_equal(ex.to_host(b), x[heads])


@pytest.mark.parametrize("dtype,n", [(np.uint32, 16_383), (np.uint32, 16_384), (np.uint32, 524_289),
                                     (np.uint32, (1 << 24) + 3), (np.int64, 131_073),
                                     (np.float64, 2_100_000), (np.float32, 600_000)])
def test_search_by_lines_levels(ex, dtype, n):
    # Sources that need from zero to seven line levels below the
    # shared-memory tree (its size just under and over a complete tree), with
    # partial last lines, against the oracle; an unaligned slice of the same
    # source takes the two-level binary search and must agree; so must the
    # binary search chosen through the tuner.
    from massively_b200 import tune, vector
    rng = np.random.default_rng(n)
    if np.dtype(dtype).kind == "f":
        src = np.sort(rng.normal(size=n).astype(dtype))
        vals = rng.normal(size=50_000).astype(dtype)
        vals[:100] = src[rng.integers(0, n, 100)]
        vals[100] = src[0]
        vals[101] = src[-1]
    else:
        src = np.sort(rng.integers(0, 1 << 20, n).astype(dtype))  # many duplicates
        vals = rng.integers(0, (1 << 20) + 5, 50_000).astype(dtype)
    ds, dv = ex.to_device(src), ex.to_device(vals)
    lo = ex.to_host(vector.lower_bound(ex, ds, dv))
    hi = ex.to_host(vector.upper_bound(ex, ds, dv))
    np.testing.assert_array_equal(lo, orc.lower_bound(src, vals))
    np.testing.assert_array_equal(hi, orc.upper_bound(src, vals))
    sl = ds.slice(1, n)
    np.testing.assert_array_equal(ex.to_host(vector.lower_bound(ex, sl, dv)),
                                  orc.lower_bound(src[1:], vals))
    tune.set_config(ex, "search", 1)
    try:
        np.testing.assert_array_equal(ex.to_host(vector.upper_bound(ex, ds, dv)), hi)
    finally:
        tune.set_config(ex, "search", -1)
