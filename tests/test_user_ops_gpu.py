"""User operators compiled at run time: reduce, inclusive / exclusive scan
and map through NVRTC-compiled kernels, exactly against sequential folds
(small sizes, pure Python where the operator has no numpy form), including
a non-commutative associative operator (composition of affine maps packed
in u64) that checks the scans keep operand order."""
import numpy as np
import pytest

from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu

SAT_ADD = "__device__ T sat_add(T a, T b) { T s = a + b; return s < a ? (T)~0u : s; }"
# (m, c) packed as m | c << 32: x -> m * x + c (mod 2^32); compose(a, b)
# applies a, then b.
COMPOSE = """
__device__ T compose(T a, T b) {
  unsigned am = (unsigned)a, ac = (unsigned)(a >> 32);
  unsigned bm = (unsigned)b, bc = (unsigned)(b >> 32);
  unsigned m = am * bm, c = bm * ac + bc;
  return (T)m | ((T)c << 32);
}
"""


def _compose(a, b):
    am, ac = a & 0xFFFFFFFF, a >> 32
    bm, bc = b & 0xFFFFFFFF, b >> 32
    return ((am * bm) & 0xFFFFFFFF) | ((((bm * ac) + bc) & 0xFFFFFFFF) << 32)


@pytest.fixture(scope="module")
def ex():
    return executor()


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 100_003, 1 << 22])
def test_user_reduce_saturating_add(ex, n):
    from massively_b200 import op, vector
    sat = op.UserOp.binary(ex, np.uint32, SAT_ADD, "sat_add")
    x = seeded(np.uint32, n, n, hi=1 << 12)
    got = vector.reduce(ex, ex.to_device(x), np.uint32(7), sat)
    assert int(got) == min(int(x.astype(np.uint64).sum()) + 7, 0xFFFFFFFF)
    big = np.full(n, 1 << 30, np.uint32)
    got = vector.reduce(ex, ex.to_device(big), np.uint32(0), sat)
    assert int(got) == min(n << 30, 0xFFFFFFFF)


@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 4097, 100_003, 600_001])
def test_user_scans_keep_operand_order(ex, n):
    from massively_b200 import op, vector
    comp = op.UserOp.binary(ex, np.uint64, COMPOSE, "compose")
    rng = np.random.default_rng(n)
    m = rng.integers(1, 1 << 32, n, dtype=np.uint64)
    c = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    x = (m | (c << np.uint64(32))).astype(np.uint64)
    d = ex.to_device(x)
    inc = ex.to_host(vector.inclusive_scan(ex, d, comp))
    init = (3 | (5 << 32))
    exc = ex.to_host(vector.exclusive_scan(ex, d, np.uint64(init), comp))
    xs = [int(v) for v in x]
    acc = None
    want_inc = np.empty(n, np.uint64)
    want_exc = np.empty(n, np.uint64)
    for i, v in enumerate(xs):
        want_exc[i] = init if acc is None else _compose(init, acc)
        acc = v if acc is None else _compose(acc, v)
        want_inc[i] = acc
    np.testing.assert_array_equal(inc, want_inc)
    np.testing.assert_array_equal(exc, want_exc)


def test_user_map_and_lazy_input(ex):
    from massively_b200 import lazy, op, vector
    bucket = op.UserOp.map(ex, np.float32, np.int32,
                           "__device__ Out bucket(In x) { return (Out)floorf(x * 4.0f); }",
                           "bucket")
    x = seeded(np.float32, 100_003, 4)
    got = ex.to_host(vector.map(ex, ex.to_device(x), bucket))
    np.testing.assert_array_equal(got, np.floor(x * np.float32(4)).astype(np.int32))
    sq = op.UserOp.map(ex, np.uint32, np.uint64,
                       "__device__ Out sq(In x) { return (Out)x * x; }", "sq")
    got = ex.to_host(vector.map(ex, lazy.counting(0).take(70_001), sq))
    np.testing.assert_array_equal(got, np.arange(70_001, dtype=np.uint64) ** 2)


def test_user_op_errors(ex):
    from massively_b200 import op, vector
    from massively_b200.runtime import Error
    sat = op.UserOp.binary(ex, np.uint32, SAT_ADD, "sat_add")
    d = ex.to_device(np.arange(10, dtype=np.uint32))
    with pytest.raises(Error):  # a map handle where a binary operator is expected
        m = op.UserOp.map(ex, np.uint32, np.uint32, "__device__ Out f(In x) { return x; }", "f")
        ex.sync()
        import ctypes as C
        from massively_b200 import _native as N
        from massively_b200.runtime import check
        out = ex.alloc(np.uint32, 10)
        check(N.lib().mb_inclusive_scan_user(ex.handle, C.byref(d.to_src()), m.handle,
                                             out.to_col()))
    assert int(vector.reduce(ex, d, np.uint32(0), sat)) == 45


# ------------------------------------------------------- user comparators --

BY_MOD = "__device__ bool by_mod(T a, T b) { return (a % 1000u) < (b % 1000u); }"
DESC = "__device__ bool desc(T a, T b) { return b < a; }"
BY_HIGH = "__device__ bool by_high(T a, T b) { return (a >> 32) < (b >> 32); }"


@pytest.mark.parametrize("n", [1, 2, 1023, 1024, 1025, 4097, 100_003, 1 << 20])
def test_user_comparator_sort_is_stable(ex, n):
    """vector::sort / sort_by_key under a user comparator with many ties
    (keys compared mod 1000): the stable order, values carried."""
    from massively_b200 import lazy, op, vector, zip2
    less = op.UserOp.predicate(ex, np.uint32, BY_MOD, "by_mod")
    keys = seeded(np.uint32, n, 40)
    want = np.argsort(keys % 1000, kind="stable")
    dk = ex.to_device(keys)
    np.testing.assert_array_equal(ex.to_host(vector.sort(ex, dk, less)), keys[want])
    vals = zip2(ex.to_device(np.arange(n, dtype=np.uint32)), lazy.counting(7).take(n))
    a, b = vector.sort_by_key(ex, dk, vals, less).into_columns()
    np.testing.assert_array_equal(ex.to_host(a), want.astype(np.uint32))
    np.testing.assert_array_equal(ex.to_host(b), (want + 7).astype(np.uint32))


@pytest.mark.parametrize("dtype,src,name,pred", [(np.float64, DESC, "desc", "greater"),
                                                 (np.int32, DESC, "desc", "greater")])
def test_user_comparator_matches_builtin_order(ex, orc, dtype, src, name, pred):
    from massively_b200 import op, vector
    less = op.UserOp.predicate(ex, dtype, src, name)
    x = seeded(dtype, 300_007, 41)
    got = ex.to_host(vector.sort_by_key(ex, ex.to_device(x),
                                        ex.to_device(np.arange(x.size, dtype=np.uint32)), less))
    np.testing.assert_array_equal(got, orc.sort_perm(x, pred))


def test_user_comparator_on_packed_u64(ex):
    """Only the high halves order the items; the low halves show the
    input order of ties."""
    from massively_b200 import op, vector
    less = op.UserOp.predicate(ex, np.uint64, BY_HIGH, "by_high")
    hi = seeded(np.uint32, 50_000, 42) % np.uint32(50)
    x = (hi.astype(np.uint64) << np.uint64(32)) | np.arange(hi.size, dtype=np.uint64)
    got = ex.to_host(vector.sort(ex, ex.to_device(x), less))
    np.testing.assert_array_equal(got, x[np.argsort(hi, kind="stable")])
