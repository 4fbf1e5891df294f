"""reduce, copy_where / remove_where / partition, gather / scatter, copy and
fill: CUDA path vs the oracle (bit-exact for integers, bounded for floats)."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, fp_bound, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


# ------------------------------------------------------------------ reduce --

def test_reduce_known_answers(ex):
    from massively_b200 import op, vector
    for case in K.REDUCE:
        assert vector.reduce(ex, ex.to_device(case["x"]), case["init"], op.Add) == case["want"]


@pytest.mark.parametrize("n", K.ORACLE_LENGTHS + [4095, 4096, 4097, 1 << 20, 5_000_011])
@pytest.mark.parametrize("dtype", [np.uint32, np.int32, np.uint64, np.int64, np.uint8, np.int16])
@pytest.mark.parametrize("opname", ["add", "min", "max", "xor", "and", "or"])
def test_integer_reduce_bit_exact(ex, n, dtype, opname):
    from massively_b200 import op, vector
    x = seeded(dtype, n, seed=n + 3)
    init = dtype(7)
    got = vector.reduce(ex, ex.to_device(x), init, op.reduction(opname))
    assert got == orc.reduce(x, opname, init)


def test_reduce_u32_widened_to_u64(ex):
    # configuration-1 reduce: 2^20 u32 keys, u64 accumulator via a lazy cast.
    from massively_b200 import lazy, op, vector
    n = 1 << 20
    x = orc.uniform_u32(0, 0xFFFFFFFF, 0, n)
    got = vector.reduce(ex, lazy.cast(ex.to_device(x), np.uint64), np.uint64(0), op.Add)
    assert int(got) == int(x.astype(np.uint64).sum())
    assert int(got) == int(orc.reduce(x.astype(np.uint64), "add", 0))


@pytest.mark.parametrize("n", [1, 1000, 1 << 20, 1 << 24])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_float_reduce_bound_and_determinism(ex, n, dtype):
    from massively_b200 import op, vector
    x = seeded(dtype, n, seed=8)
    d = ex.to_device(x)
    got = vector.reduce(ex, d, dtype(0), op.Add)
    exact = float(x.astype(np.float64).sum())
    assert abs(float(got) - exact) <= fp_bound(x) + 1e-30
    assert vector.reduce(ex, d, dtype(0), op.Add) == got  # same bits run to run
    assert vector.reduce(ex, d, dtype(np.inf), op.Min) == orc.reduce(x, "min", dtype(np.inf))
    assert vector.reduce(ex, d, dtype(-np.inf), op.Max) == orc.reduce(x, "max", dtype(-np.inf))


def test_reduce_lazy_and_empty(ex):
    from massively_b200 import lazy, op, vector
    assert vector.reduce(ex, ex.to_device(np.zeros(0, np.uint32)), np.uint32(9), op.Add) == 9
    n = 123_457
    got = vector.reduce(ex, lazy.counting(1).take(n), np.uint32(0), op.Add)
    assert got == np.uint32((n * (n + 1) // 2) & 0xFFFFFFFF)
    x = seeded(np.uint32, n, 4)
    got = vector.reduce(ex, lazy.map(ex.to_device(x), op.IsEven), np.uint32(0), op.Add)
    assert got == int(((x & 1) == 0).sum())
    assert vector.reduce(ex, ex.to_device(x), np.uint32(5), op.TakeLeft) == 5
    assert vector.reduce(ex, ex.to_device(x), np.uint32(5), op.TakeRight) == x[-1]


# -------------------------------------------------------------- selection --

def test_selection_known_answers(ex):
    from massively_b200 import op, vector, zip3
    for case in K.SELECT:
        fn = vector.copy_where if case["kind"] == "copy_where" else vector.remove_where
        got = fn(ex, ex.to_device(case["x"]), ex.to_device(case["stencil"]))
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    r = K.COPY_WHERE_ROWS
    got = vector.copy_where(ex, zip3(*[ex.to_device(c) for c in r["cols"]]),
                            ex.to_device(r["stencil"]))
    for g, w in zip(got.into_columns(), r["want"]):
        np.testing.assert_array_equal(ex.to_host(g), w)
    for case in K.PARTITION:
        out, b = vector.partition(ex, ex.to_device(case["x"]), op.unary(case["pred"]))
        assert b == case["boundary"]
        np.testing.assert_array_equal(ex.to_host(out), case["want"])


@pytest.mark.parametrize("n", K.ORACLE_LENGTHS + [4095, 4096, 4097, 1 << 20, 3_000_017])
@pytest.mark.parametrize("density", ["half", "sparse", "none", "all"])
def test_copy_where_fused_predicate(ex, n, density):
    from massively_b200 import lazy, op, vector
    x = seeded(np.uint32, n, seed=n + 1)
    if density == "sparse":
        x = np.where(x % 97 == 0, x & ~np.uint32(1), x | 1).astype(np.uint32)
    elif density == "none":
        x = x | 1
    elif density == "all":
        x = x & ~np.uint32(1)
    d = ex.to_device(x)
    st = orc.flags(x, "is_even")
    got = vector.copy_where(ex, d, lazy.map(d, op.IsEven))
    np.testing.assert_array_equal(ex.to_host(got), orc.copy_where(x, st))
    got = vector.remove_where(ex, d, lazy.map(d, op.IsEven))
    np.testing.assert_array_equal(ex.to_host(got), orc.remove_where(x, st))
    # a materialised stencil column of arbitrary non-zero flags
    flags = (seeded(np.uint32, n, 77) % 5).astype(np.uint32)
    got = vector.copy_where(ex, d, ex.to_device(flags))
    np.testing.assert_array_equal(ex.to_host(got), orc.copy_where(x, flags))


@pytest.mark.parametrize("n", [0, 33, 4097, 100_003])
def test_copy_where_multi_column_types(ex, n):
    from massively_b200 import vector, zip4
    cols = [seeded(np.uint32, n, 1), seeded(np.float32, n, 2), seeded(np.int64, n, 3),
            seeded(np.uint8, n, 4)]
    flags = (seeded(np.uint32, n, 5) & 1).astype(np.uint32)
    got = vector.copy_where(ex, zip4(*[ex.to_device(c) for c in cols]), ex.to_device(flags))
    want = orc.copy_where(cols, flags)
    for g, w in zip(got.into_columns(), want):
        np.testing.assert_array_equal(ex.to_host(g).view(np.uint8), w.view(np.uint8))


@pytest.mark.parametrize("n", [1, 257, 70_001, 1 << 20])
@pytest.mark.parametrize("pred", ["is_even", "is_odd", "is_true"])
def test_partition_stable(ex, n, pred):
    from massively_b200 import op, vector
    x = (seeded(np.uint32, n, 6) % 10).astype(np.uint32)
    out, b = vector.partition(ex, ex.to_device(x), op.unary(pred))
    want, wb = orc.partition(x, pred)
    assert b == wb
    np.testing.assert_array_equal(ex.to_host(out), want)


def test_selection_pipeline_device_length(ex):
    # copy_where's device count feeds a second copy_where without a host sync.
    from massively_b200 import lazy, op, vector
    n = 200_003
    x = seeded(np.uint32, n, 9)
    d = ex.to_device(x)
    a = vector.copy_where(ex, d, lazy.map(d, op.IsEven))
    b = vector.copy_where(ex, a, lazy.map(a, op.IsTrue))
    ax = orc.copy_where(x, orc.flags(x, "is_even"))
    np.testing.assert_array_equal(ex.to_host(b), orc.copy_where(ax, orc.flags(ax, "is_true")))


# --------------------------------------------------------- gather/scatter --

def test_gather_scatter_known_answers(ex):
    from massively_b200 import vector
    for case in K.GATHER:
        if case["stencil"] is None:
            got = vector.gather(ex, ex.to_device(case["values"]), ex.to_device(case["idx"]))
        else:
            got = ex.to_device(case["out"])
            vector.gather_where(ex, ex.to_device(case["values"]), ex.to_device(case["idx"]),
                                ex.to_device(case["stencil"]), got)
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    for case in K.SCATTER:
        out = ex.to_device(case["out"])
        if case["stencil"] is None:
            vector.scatter(ex, ex.to_device(case["values"]), ex.to_device(case["idx"]), out)
        else:
            vector.scatter_where(ex, ex.to_device(case["values"]), ex.to_device(case["idx"]),
                                 ex.to_device(case["stencil"]), out)
        np.testing.assert_array_equal(ex.to_host(out), case["want"], err_msg=case["src"])
    ex.sync()


@pytest.mark.parametrize("n", [0, 1, 4097, 1 << 20])
@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32, np.float64])
def test_gather_scatter_permutations(ex, n, dtype):
    from massively_b200 import lazy, vector
    vals = seeded(dtype, n, 3)
    idx = orc.sort_perm(seeded(np.uint32, n, 4))  # a permutation
    got = vector.gather(ex, ex.to_device(vals), ex.to_device(idx))
    np.testing.assert_array_equal(ex.to_host(got).view(np.uint8), vals[idx].view(np.uint8))
    out = ex.zeros(dtype, n)
    vector.scatter(ex, ex.to_device(vals), ex.to_device(idx), out)
    np.testing.assert_array_equal(ex.to_host(out).view(np.uint8),
                                  orc.scatter(vals, idx, np.zeros(n, dtype)).view(np.uint8))
    # reverse indices (the scale tests' indices_for)
    rev = np.arange(n, dtype=np.uint32)[::-1].copy()
    got = vector.gather(ex, ex.to_device(vals), lazy.reverse(lazy.counting(0).take(n))
                        if n else ex.to_device(rev))
    np.testing.assert_array_equal(ex.to_host(got).view(np.uint8), vals[rev].view(np.uint8))
    ex.sync()


def test_copy_fill_and_views(ex):
    from massively_b200 import lazy, op, vector
    n = 10_007
    x = seeded(np.int32, n, 2)
    d = ex.to_device(x)
    out = ex.alloc(np.int32, n)
    vector.fill(ex, np.int32(-7), out)
    assert (ex.to_host(out) == -7).all()
    np.testing.assert_array_equal(ex.to_host(vector.map(ex, d, op.Negate)), -x)
    np.testing.assert_array_equal(ex.to_host(vector.map(ex, d, op.Abs)), np.abs(x))
    np.testing.assert_array_equal(ex.to_host(vector.map(ex, lazy.repeat_each(d, 3), op.Identity)),
                                  np.repeat(x, 3))
    np.testing.assert_array_equal(ex.to_host(vector.map(ex, lazy.tile(d, 2), op.Identity)),
                                  np.tile(x, 2))
    np.testing.assert_array_equal(ex.to_host(vector.map(ex, lazy.stride(3, 5).take(9),
                                                        op.Identity)),
                                  np.arange(9, dtype=np.uint32) * 5 + 3)
    np.testing.assert_array_equal(
        ex.to_host(vector.adjacent_difference(ex, ex.to_device(np.array([1, 3, 6, 10], np.uint32)),
                                              op.Add)), [1, 4, 9, 16])
    np.testing.assert_array_equal(ex.to_host(vector.reverse(ex, d)), x[::-1])


def test_random_streams_match_oracle(ex):
    import massively_b200 as mb
    from massively_b200 import _native as N
    n = 100_000
    out = ex.alloc(np.uint32, n)
    mb.runtime.check(N.lib().mb_random_uniform_u32(ex.handle, 10, 20, 123, 5, out.to_col()))
    np.testing.assert_array_equal(ex.to_host(out), orc.uniform_u32(10, 20, 123, n, offset=5))
    out64 = ex.alloc(np.uint64, n)
    mb.runtime.check(N.lib().mb_random_uniform_u64(ex.handle, 0, 2**64 - 1, 2, 0,
                                                   out64.to_col()))
    np.testing.assert_array_equal(ex.to_host(out64), orc.uniform_u64(0, 2**64 - 1, 2, n))


# ----------------------------------------------- replace / transform where --

def test_replace_where_known_answers_and_seeded(ex):
    """vector::replace_where: the reference's doctest and owned-value test,
    then seeded stencils over every element width and a zipped output."""
    from massively_b200 import lazy, op, vector, zip2
    for case in K.REPLACE_WHERE:
        out = ex.to_device(case["out"])
        vector.replace_where(ex, np.uint32(case["value"]), ex.to_device(case["stencil"]), out)
        np.testing.assert_array_equal(ex.to_host(out), case["want"], err_msg=case["src"])
    for dtype in (np.uint8, np.int16, np.uint32, np.float32, np.int64, np.float64):
        n = 70_001
        base = seeded(dtype, n, 5)
        st = (seeded(np.uint32, n, 6) % 3 == 0).astype(np.uint32)
        value = np.array([7], dtype)[0]
        out = ex.to_device(base)
        vector.replace_where(ex, value, ex.to_device(st), out)
        np.testing.assert_array_equal(ex.to_host(out).view(np.uint8),
                                      orc.replace_where(value, st, base).view(np.uint8))
    # zipped output, lazy stencil (is_odd over a column)
    n = 4099
    a, b = seeded(np.uint32, n, 7), seeded(np.float32, n, 8)
    key = seeded(np.uint32, n, 9)
    oa, ob = ex.to_device(a), ex.to_device(b)
    vector.replace_where(ex, (np.uint32(5), np.float32(-1.5)),
                         lazy.map(ex.to_device(key), op.IsOdd), zip2(oa, ob))
    st = (key & 1).astype(np.uint32)
    np.testing.assert_array_equal(ex.to_host(oa), orc.replace_where(5, st, a))
    np.testing.assert_array_equal(ex.to_host(ob), orc.replace_where(np.float32(-1.5), st, b))


def test_transform_where_seeded_and_errors(ex):
    """vector::transform_where with built-in unary operators: op(x) where the
    stencil is set, the output kept elsewhere; length errors as massively's
    (core/selection.rs:538-551)."""
    from massively_b200 import op, vector
    from massively_b200.runtime import LengthMismatch
    for dtype, unary, host_op in [(np.int32, op.Negate, lambda x: -x),
                                  (np.uint32, op.BitNot, lambda x: ~x),
                                  (np.float64, op.Abs, np.abs),
                                  (np.uint64, op.IsEven, lambda x: (x & 1) == 0)]:
        n = 100_003
        x = seeded(dtype, n, 10)
        st = (seeded(np.uint32, n, 11) & 1).astype(np.uint32)
        out_dt = np.uint32 if unary is op.IsEven else dtype
        base = seeded(out_dt, n, 12)
        out = ex.to_device(base)
        vector.transform_where(ex, ex.to_device(x), unary, ex.to_device(st), out)
        want = orc.transform_where(x, host_op, st, base)
        np.testing.assert_array_equal(ex.to_host(out).view(np.uint8), want.view(np.uint8))
    d3 = ex.to_device(np.arange(3, dtype=np.uint32))
    d4 = ex.to_device(np.arange(4, dtype=np.uint32))
    with pytest.raises(LengthMismatch) as e:
        vector.transform_where(ex, d3, op.Identity, d4, ex.to_device(np.zeros(3, np.uint32)))
    assert (e.value.left, e.value.right) == (3, 4)
    with pytest.raises(LengthMismatch) as e:
        vector.transform_where(ex, d3, op.Identity, d3, ex.to_device(np.zeros(4, np.uint32)))
    assert (e.value.left, e.value.right) == (3, 4)
    with pytest.raises(LengthMismatch) as e:
        vector.replace_where(ex, np.uint32(1), d3, ex.to_device(np.zeros(4, np.uint32)))
    assert (e.value.left, e.value.right) == (3, 4)
