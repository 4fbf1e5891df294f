"""scatter_reduce: the CUDA path against the oracle (restating
massively/src/api/algorithm/scatter.rs:332-420), exactly for every integer op
and type and for float MIN / MAX, within the association bound for float ADD;
on the reference's doctest and unit tests (multi-column rows), heavy and
sparse collisions, identity and non-identity inits, narrow columns, lazy
values and indices, and the bounds check."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu

IDENTITY = {"add": 0, "mul": 1, "and": -1, "or": 0, "xor": 0}


@pytest.fixture(scope="module")
def ex():
    return executor()


def test_known_answers(ex):
    from massively_b200 import Zip, vector
    for case in K.SCATTER_REDUCE:
        vals = [ex.to_device(v) for v in case["values"]]
        outs = [ex.to_device(o) for o in case["output"]]
        v = Zip(*vals) if len(vals) > 1 else vals[0]
        o = Zip(*outs) if len(outs) > 1 else outs[0]
        init = tuple(case["init"]) if len(vals) > 1 else case["init"][0]
        vector.scatter_reduce(ex, v, ex.to_device(case["indices"]), init, case["op"], o)
        for got, want in zip(outs, case["want"]):
            np.testing.assert_array_equal(ex.to_host(got), want, err_msg=case["src"])


def _ident(op, dtype):
    dt = np.dtype(dtype)
    if op == "min":
        return np.inf if dt.kind == "f" else np.iinfo(dt).max
    if op == "max":
        return -np.inf if dt.kind == "f" else np.iinfo(dt).min
    if op == "and":
        return np.array(-1).astype(dt) if dt.kind != "f" else None
    return IDENTITY[op]


def _inputs(dtype, n, nout, seed):
    dt = np.dtype(dtype)
    idx = seeded(np.uint32, n, seed, hi=nout - 1)
    if dt.kind == "f":
        v = np.round(seeded(np.float32, n, seed + 1) * 8).astype(dt)
        out = np.round(seeded(np.float32, nout, seed + 2) * 8).astype(dt)
    else:
        lo, hi = (0, 1000) if dt.kind == "u" else (-500, 500)
        v = (seeded(np.uint32, n, seed + 1, hi=hi - lo) .astype(np.int64) + lo).astype(dt)
        out = (seeded(np.uint32, nout, seed + 2, hi=hi - lo).astype(np.int64) + lo).astype(dt)
    return v, idx, out


INT_TYPES = [np.uint8, np.int16, np.uint32, np.int32, np.uint64, np.int64]


@pytest.mark.parametrize("dtype", INT_TYPES)
@pytest.mark.parametrize("op", ["add", "mul", "min", "max", "and", "or", "xor"])
@pytest.mark.parametrize("n,nout", [(1, 1), (1000, 1), (100_003, 37), (100_003, 70_001),
                                    (1 << 20, 1 << 22)])
def test_integer_ops_exact(ex, dtype, op, n, nout):
    from massively_b200 import vector
    v, idx, out = _inputs(dtype, n, nout, n + nout)
    if op == "mul":
        v = (np.abs(v.astype(np.int64)) % 3 + 1).astype(dtype)  # keep products varied
    d = ex.to_device(out)
    vector.scatter_reduce(ex, ex.to_device(v), ex.to_device(idx), _ident(op, dtype), op, d)
    np.testing.assert_array_equal(ex.to_host(d),
                                  orc.scatter_reduce(v, idx, _ident(op, dtype), op, out))


@pytest.mark.parametrize("dtype", [np.uint8, np.int32, np.uint64, np.float32, np.float64])
@pytest.mark.parametrize("op", ["add", "min", "max"])
def test_non_identity_init(ex, dtype, op):
    from massively_b200 import vector
    n, nout = 50_000, 30_011  # some destinations receive nothing
    v, idx, out = _inputs(dtype, n, nout, 5)
    init = {"add": 3, "min": 4, "max": 2}[op]
    d = ex.to_device(out)
    vector.scatter_reduce(ex, ex.to_device(v), ex.to_device(idx), init, op, d)
    np.testing.assert_array_equal(ex.to_host(d), orc.scatter_reduce(v, idx, init, op, out))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", ["min", "max", "mul"])
def test_float_cas_ops_exact(ex, dtype, op):
    from massively_b200 import vector
    n, nout = 200_003, 1009
    v, idx, out = _inputs(dtype, n, nout, 9)
    if op == "mul":
        v = np.where(seeded(np.uint32, n, 3, hi=1) == 0, 1.0, -1.0).astype(dtype)  # exact products
    d = ex.to_device(out)
    vector.scatter_reduce(ex, ex.to_device(v), ex.to_device(idx), _ident(op, dtype), op, d)
    np.testing.assert_array_equal(ex.to_host(d),
                                  orc.scatter_reduce(v, idx, _ident(op, dtype), op, out))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n,nout", [(1 << 20, 17), (1 << 20, 1 << 18)])
def test_float_add_within_bound(ex, dtype, n, nout):
    """Proposals of a destination arrive in any order: each result is within
    k * eps * (|out| + sum |v|) of the exact sum, k = proposals + 1."""
    from massively_b200 import vector
    idx = seeded(np.uint32, n, 21, hi=nout - 1)
    v = seeded(np.float32, n, 22).astype(dtype)
    out = seeded(np.float32, nout, 23).astype(dtype)
    d = ex.to_device(out)
    vector.scatter_reduce(ex, ex.to_device(v), ex.to_device(idx), 0.0, "add", d)
    got = ex.to_host(d).astype(np.float64)
    exact = out.astype(np.float64).copy()
    np.add.at(exact, idx, v.astype(np.float64))
    absum = np.abs(out).astype(np.float64)
    np.add.at(absum, idx, np.abs(v).astype(np.float64))
    k = np.bincount(idx, minlength=nout) + 1
    eps = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
    assert np.all(np.abs(got - exact) <= k * eps * absum + 1e-300)


def test_lazy_values_and_indices(ex):
    from massively_b200 import lazy, vector
    nout, n = 1000, 1_000_003
    out = np.zeros(nout, np.uint64)
    d = ex.to_device(out)
    # values 0..n-1 (a cast counting view) into destination i % nout (a tile view)
    values = lazy.cast(lazy.counting(0).take(n), np.uint64)
    indices = lazy.tile(ex.to_device(np.arange(nout, dtype=np.uint32)), n // nout + 1).take(n)
    vector.scatter_reduce(ex, values, indices, 0, "add", d)
    vals = np.arange(n, dtype=np.uint64)
    idx = (np.arange(n) % nout).astype(np.uint32)
    np.testing.assert_array_equal(ex.to_host(d), orc.scatter_reduce(vals, idx, 0, "add", out))


def test_errors():
    import massively_b200 as mb
    from massively_b200 import vector
    from massively_b200.runtime import Error, LengthMismatch
    ex2 = executor()
    v = ex2.to_device(np.array([1, 2, 3], np.uint32))
    o = ex2.to_device(np.zeros(4, np.uint32))
    with pytest.raises(LengthMismatch):
        vector.scatter_reduce(ex2, v, ex2.to_device(np.array([0, 1], np.uint32)), 0, "add", o)
    with pytest.raises(Error):
        vector.scatter_reduce(ex2, v, ex2.to_device(np.array([0, 1, 2], np.uint32)), 0,
                              "take_left", o)
    with pytest.raises(Error):  # element types differ
        vector.scatter_reduce(ex2, v, ex2.to_device(np.array([0, 1, 2], np.uint32)), 0, "add",
                              ex2.to_device(np.zeros(4, np.int32)))
    # an index past the output is skipped and reported at the next sync
    vector.scatter_reduce(ex2, v, ex2.to_device(np.array([0, 9, 2], np.uint32)), 0, "add", o)
    with pytest.raises(mb.runtime.Launch):
        ex2.sync()
    np.testing.assert_array_equal(ex2.to_host(o), [1, 0, 3, 0])
    ex2.sync()  # the status word was cleared
