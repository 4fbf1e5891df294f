"""Predicates, first-index searches and extrema: the CUDA path against the
oracle (restating massively's verification/oracle/src/vector.rs:176-218,
317-378, 428-481 and massively/src/core/predicate.rs:111-127), exactly, on the
reference's doctests and unit tests, on seeded inputs with planted hits at
tile edges, on every element type and order, on NaNs, empty and ragged
inputs, lazy views, device-length inputs and device-resident results."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu

NONE = 0xFFFFFFFF
SIZES = [0, 1, 2, 2047, 2048, 2049, 100_003, 1 << 22]


@pytest.fixture(scope="module")
def ex():
    return executor()


def _dev_call(ex, fn, args, kwargs=None):
    from massively_b200 import vector
    return getattr(vector, fn)(ex, *args, **(kwargs or {}))


def test_known_answers(ex):
    from massively_b200 import op
    for case in K.PREDICATES:
        a = ex.to_device(case["a"])
        arg = case["arg"]
        if arg in ("less", "equal"):
            arg = {"less": op.Less, "equal": op.Equal}[arg]
        args = [a, ex.to_device(case["b"]), arg] if "b" in case else [a, arg]
        assert _dev_call(ex, case["fn"], args) == case["want"], case["src"]


def test_count_if_four_billion_lazy(ex):
    from massively_b200 import lazy, vector
    case = K.COUNT_IF_FOUR_BILLION
    x = lazy.counting(0).take(case["n"])
    assert vector.count_if(ex, x, case["pred"]) == case["want"], case["src"]


def _planted(n, seed, hits):
    """Odd values with even ones planted at `hits` (positions < n)."""
    x = (seeded(np.uint32, n, seed) | 1).astype(np.uint32)
    for h in hits:
        if 0 <= h < n:
            x[h] = 2 * (h % 1000)
    return x


@pytest.mark.parametrize("n", SIZES)
def test_find_if_planted(ex, n):
    from massively_b200 import vector
    for hits in ([], [0], [n - 1], [n // 2, n - 1], [2047, 2048, n - 2], [n // 3, n // 7]):
        x = _planted(n, n + len(hits), hits)
        d = ex.to_device(x)
        assert vector.find_if(ex, d, "is_even") == orc.find_if(x, "is_even"), hits
        assert vector.count_if(ex, d, "is_even") == orc.count_if(x, "is_even")
        assert vector.any_of(ex, d, "is_even") == orc.any_of(x, "is_even")
        assert vector.none_of(ex, d, "is_even") == orc.none_of(x, "is_even")
        assert vector.all_of(ex, d, "is_odd") == orc.all_of(x, "is_odd")
        assert vector.is_partitioned(ex, d, "is_odd") == orc.is_partitioned(x, "is_odd")


@pytest.mark.parametrize("dtype", [np.int8, np.uint16, np.int32, np.uint64, np.int64,
                                   np.float32, np.float64])
@pytest.mark.parametrize("pred", ["is_true", "is_false", "is_negative", "is_positive",
                                  "is_even"])
def test_find_if_types(ex, dtype, pred):
    from massively_b200 import vector
    if np.dtype(dtype).kind == "f" and pred == "is_even":
        pytest.skip("IS_EVEN takes integer items")
    n = 70_001
    rng = np.random.default_rng(7)
    x = rng.integers(1, 50, n).astype(dtype)
    x[rng.integers(0, n, 3)] = 0
    if np.dtype(dtype).kind in "if":
        x[n - 5] = -3
    d = ex.to_device(x)
    assert vector.find_if(ex, d, pred) == orc.find_if(x, pred)
    assert vector.count_if(ex, d, pred) == orc.count_if(x, pred)
    assert vector.is_partitioned(ex, d, pred) == orc.is_partitioned(x, pred)


def test_is_partitioned_shapes(ex):
    from massively_b200 import vector
    for n in [0, 1, 2, 2049, 100_003]:
        for cut in sorted({0, 1, n // 2, n}):
            x = np.ones(n, np.uint32)
            x[:cut] = 2  # passing (even) prefix, failing suffix
            d = ex.to_device(x)
            assert vector.is_partitioned(ex, d, "is_even") is True
            if n > cut + 1:
                x[n - 1] = 4  # a passing item after the failing run
                assert vector.is_partitioned(ex, ex.to_device(x), "is_even") == \
                    orc.is_partitioned(x, "is_even") is False


@pytest.mark.parametrize("n", SIZES)
def test_adjacent_find_and_sorted_until(ex, n):
    from massively_b200 import op, vector
    base = np.arange(n, dtype=np.int64) * 3
    for plant in [None, 0, n // 2, n - 2, 2047]:
        x = base.copy()
        if plant is not None and 0 <= plant < n - 1:
            x[plant + 1] = x[plant]          # an equal neighbour
        d = ex.to_device(x)
        assert vector.adjacent_find(ex, d) == orc.adjacent_find(x)
        y = base.copy()
        if plant is not None and 0 <= plant < n - 1:
            y[plant + 1] = y[plant] - 1      # the first descent
        dy = ex.to_device(y)
        assert vector.is_sorted_until(ex, dy) == orc.is_sorted_until(y)
        assert vector.is_sorted(ex, dy) == orc.is_sorted(y)
        assert vector.is_sorted_until(ex, dy, op.Greater) == orc.is_sorted_until(y, "greater")


def test_sorted_until_floats_and_orders(ex):
    from massively_b200 import op, vector
    x = np.sort(seeded(np.float32, 50_000, 3))
    x[100] = -0.0
    x[101] = 0.0  # -0 == +0 under `<`, ordered under the total order
    x.sort()
    x[30_000] = np.nan
    d = ex.to_device(x)
    for less, name in [(op.Less, "less"), (op.Greater, "greater"), (op.TotalLess, "total_less")]:
        assert vector.is_sorted_until(ex, d, less) == orc.is_sorted_until(x, name), name


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 5), (5, 0), (3, 3), (2049, 2049), (2049, 4000),
                                   (100_003, 100_000), (1 << 22, 1 << 22)])
def test_mismatch_equal_lexicographic(ex, na, nb):
    from massively_b200 import op, vector
    common = seeded(np.uint32, max(na, nb), na + nb, hi=1000)
    for diff in [None, 0, min(na, nb) - 1, min(na, nb) // 2, 2048]:
        a, b = common[:na].copy(), common[:nb].copy()
        if diff is not None and 0 <= diff < min(na, nb):
            b[diff] += 1
        da, db = ex.to_device(a), ex.to_device(b)
        assert vector.mismatch(ex, da, db) == orc.mismatch(a, b), diff
        assert vector.equal(ex, da, db) == orc.equal(a, b), diff
        assert vector.lexicographical_compare(ex, da, db) == orc.lexicographical_compare(a, b)
        assert vector.lexicographical_compare(ex, db, da) == orc.lexicographical_compare(b, a)
        assert vector.lexicographical_compare(ex, da, db, op.Greater) == \
            orc.lexicographical_compare(a, b, "greater")


def test_float_equality_semantics(ex):
    from massively_b200 import vector
    a = np.array([1.0, -0.0, np.nan, 2.0], np.float32)
    b = np.array([1.0, 0.0, np.nan, 2.0], np.float32)
    da, db = ex.to_device(a), ex.to_device(b)
    assert vector.mismatch(ex, da, db) == orc.mismatch(a, b) == 2  # NaN != NaN
    assert vector.equal(ex, da, da) is False
    x = np.array([np.nan, np.nan, 0.0, -0.0], np.float32)
    assert vector.adjacent_find(ex, ex.to_device(x)) == orc.adjacent_find(x) == 2


@pytest.mark.parametrize("n", [0, 1, 4, 2049, 100_003, 1 << 21])
@pytest.mark.parametrize("m", [0, 1, 7, 2048, 3000])
def test_find_first_of(ex, n, m):
    from massively_b200 import vector
    x = seeded(np.uint32, n, n + 1, hi=1 << 30)
    needles = seeded(np.uint32, m, m + 2, lo=(1 << 30) + 1)  # absent from x
    if m:
        for pos in [n - 1, n // 2, 2048 if n > 2048 else n - 1]:
            if 0 <= pos < n:
                x[pos] = needles[(pos * 7) % m]
    if n > 200:
        # a small source against many needles keeps the oracle's n * m loop short
        x = x[: 200 if m > 7 else n]
    d, dn = ex.to_device(x), ex.to_device(needles)
    assert vector.find_first_of(ex, d, dn) == orc.find_first_of(x, needles)


ORDERS = [("less", "Less"), ("greater", "Greater"), ("total_less", "TotalLess")]


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint32, np.int32, np.uint64,
                                   np.int64, np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 2, 2047, 2049, 100_003, 1 << 22])
def test_extrema_types(ex, dtype, n):
    from massively_b200 import op, vector
    rng = np.random.default_rng(n)
    if np.dtype(dtype).kind == "f":
        x = np.round(rng.normal(size=n) * 4).astype(dtype)  # many ties
    else:
        info = np.iinfo(dtype)
        x = rng.integers(max(info.min, -20), min(info.max, 20), n).astype(dtype)
    d = ex.to_device(x)
    for name, attr in ORDERS:
        less = getattr(op, attr)
        assert vector.min_element(ex, d, less) == orc.min_element(x, name), name
        assert vector.max_element(ex, d, less) == orc.max_element(x, name), name
        assert vector.minmax_element(ex, d, less) == orc.minmax_element(x, name), name


def test_extrema_empty(ex):
    from massively_b200 import vector
    d = ex.to_device(np.empty(0, np.float32))
    assert vector.min_element(ex, d) is None
    assert vector.max_element(ex, d) is None
    assert vector.minmax_element(ex, d) is None


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_extrema_nan_sequential_semantics(ex, dtype):
    from massively_b200 import op, vector
    nan = np.nan
    cases = [
        [nan, -1, -2, 5],
        [1, nan, 3, -4, -4],
        [0, -5, nan, 3, 4, 3],
        [0, -5, nan],
        [nan],
        [nan, nan, 1, 1],
        [2, nan, 1, nan, 1, 7, nan, 0, 0, 9],
    ]
    rng = np.random.default_rng(9)
    big = np.round(rng.normal(size=300_007) * 3).astype(dtype)
    for where in [[5], [150_000, 299_000], [300_006], [0, 2048, 4096]]:
        y = big.copy()
        y[where] = nan
        cases.append(y)
    for c in cases:
        x = np.asarray(c, dtype)
        d = ex.to_device(x)
        for name, attr in ORDERS:
            less = getattr(op, attr)
            assert vector.min_element(ex, d, less) == orc.min_element(x, name), (name, c)
            assert vector.max_element(ex, d, less) == orc.max_element(x, name), (name, c)
            assert vector.minmax_element(ex, d, less) == orc.minmax_element(x, name), (name, c)


def test_lazy_views(ex):
    from massively_b200 import lazy, op, vector
    x = seeded(np.int32, 100_003, 4, hi=1000)
    d = ex.to_device(x)
    r = x[::-1].copy()
    assert vector.min_element(ex, lazy.reverse(d)) == orc.min_element(r)
    assert vector.minmax_element(ex, lazy.reverse(d)) == orc.minmax_element(r)
    neg = (-x).astype(np.int32)
    assert vector.max_element(ex, lazy.map(d, op.Negate)) == orc.max_element(neg)
    assert vector.find_if(ex, lazy.map(d, op.Negate), "is_positive") == \
        orc.find_if(neg, "is_positive")
    assert vector.is_sorted_until(ex, lazy.counting(5).take(1 << 20)) == 1 << 20
    assert vector.find_if(ex, lazy.counting(1).take(10_000_001), "is_even") == 1
    assert vector.find_if(ex, lazy.stride(1, 2).take(1 << 20), "is_even") is None
    assert vector.count_if(ex, lazy.counting(0).take(1_000_001), "is_odd") == 500_000


def test_device_length_input(ex):
    """A copy_where result carries its length on the device; the searches use
    that length, not the capacity."""
    from massively_b200 import vector
    n = 200_001
    x = seeded(np.uint32, n, 12, hi=1 << 20)
    st = (x % 3 == 0).astype(np.uint32)
    kept = x[st != 0]
    sel = vector.copy_where(ex, ex.to_device(x), ex.to_device(st))
    assert vector.min_element(ex, sel) == orc.min_element(kept)
    assert vector.max_element(ex, sel) == orc.max_element(kept)
    assert vector.is_sorted_until(ex, sel) == orc.is_sorted_until(kept)
    assert vector.find_if(ex, sel, "is_odd") == orc.find_if(kept, "is_odd")


def test_device_results(ex):
    from massively_b200 import vector
    x = _planted(1 << 20, 5, [777_777])
    d = ex.to_device(x)
    out = ex.alloc(np.uint32, 2)
    assert vector.find_if(ex, d, "is_even", out=out) is None
    assert int(ex.to_host(out)[0]) == 777_777
    vector.minmax_element(ex, d, out=out)
    assert tuple(int(v) for v in ex.to_host(out)) == orc.minmax_element(x)
    vector.adjacent_find(ex, d, out=out)
    assert int(ex.to_host(out)[0]) == (orc.adjacent_find(x) if orc.adjacent_find(x) is not None
                                       else NONE)


def test_errors(ex):
    from massively_b200 import op, vector
    from massively_b200.runtime import Error
    d = ex.to_device(np.array([1.0, 2.0], np.float32))
    with pytest.raises(Error):
        vector.find_if(ex, d, "is_even")  # IS_EVEN takes integer items
    with pytest.raises(Error):
        vector.mismatch(ex, d, ex.to_device(np.array([1, 2], np.uint32)))
    with pytest.raises(Error):
        vector.min_element(ex, d, op.Equal)


def test_count_logical_length(ex):
    """vector::count (predicate.rs:49-51): the logical item count, device
    lengths included."""
    from massively_b200 import lazy, vector
    assert vector.count(ex, ex.to_device(np.array([1, 2, 3, 4], np.uint32))) == 4
    x = seeded(np.uint32, 10_001, 3)
    st = (x % 2).astype(np.uint32)
    sel = vector.copy_where(ex, ex.to_device(x), ex.to_device(st))
    assert vector.count(ex, sel) == int(st.sum())
    assert vector.count(ex, lazy.counting(0).take(77)) == 77


def test_count_of_zipped_columns_is_the_shortest_logical_length(ex):
    """A zip whose later column carries the shorter device length counts the
    rows every column holds."""
    from massively_b200 import vector
    from massively_b200.iter import Zip
    n = 5000
    a = ex.to_device(np.arange(n, dtype=np.uint32))
    b = ex.to_device(np.arange(n, dtype=np.uint32)).with_len_dev(
        ex.to_device(np.array([1234], np.uint32)).tensor)
    assert vector.count(ex, Zip(a, b)) == 1234
    assert vector.count(ex, Zip(b, a)) == 1234
