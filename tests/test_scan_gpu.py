"""Scan parity: CUDA path (through the C ABI) vs the oracle, bit-exact for
integers; floats within the association bound against an FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, fp_bound, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def test_known_answers(ex):
    from massively_b200 import op, vector
    for case in K.SCAN:
        x = ex.to_device(case["x"])
        if case["kind"] == "inclusive":
            got = vector.inclusive_scan(ex, x, op.Add)
        else:
            got = vector.exclusive_scan(ex, x, case["init"], op.Add)
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    ones = ex.to_device(np.ones(K.SCAN_ONES["n"], np.uint32))
    inc = ex.to_host(vector.inclusive_scan(ex, ones, op.Add))
    for i, v in K.SCAN_ONES["probes"].items():
        assert inc[i] == v
    exc = ex.to_host(vector.exclusive_scan(ex, ones, K.SCAN_EXCL_ONES["init"], op.Add))
    for i in K.SCAN_EXCL_ONES["probes"]:
        assert exc[i] == K.SCAN_EXCL_ONES["init"] + i
    tl = ex.to_host(vector.exclusive_scan(ex, ones.slice(0, K.SCAN_TAKE_LEFT["n"]),
                                          K.SCAN_TAKE_LEFT["init"], op.TakeLeft))
    assert (tl == K.SCAN_TAKE_LEFT["want"]).all()


@pytest.mark.parametrize("n", K.ORACLE_LENGTHS + [4095, 4096, 4097, 70_001, 1 << 20, 3_000_017])
@pytest.mark.parametrize("dtype", [np.uint32, np.int32, np.uint64, np.int64, np.uint8, np.int16])
@pytest.mark.parametrize("opname", ["add", "min", "max", "xor", "mul", "take_left"])
def test_integer_scans_bit_exact(ex, n, dtype, opname):
    from massively_b200 import op, vector
    if n > 100_000 and (opname in ("mul", "take_left") or dtype not in (np.uint32, np.uint64)):
        pytest.skip("large sizes: u32/u64 add/min/max/xor only")
    x = seeded(dtype, n, seed=n * 7 + 1)
    if opname == "mul":
        x = (x | 1).astype(dtype)
    d = ex.to_device(x)
    o = op.reduction(opname)
    got = ex.to_host(vector.inclusive_scan(ex, d, o))
    np.testing.assert_array_equal(got, orc.inclusive_scan(x, opname))
    init = dtype(5)
    got = ex.to_host(vector.exclusive_scan(ex, d, init, o))
    np.testing.assert_array_equal(got, orc.exclusive_scan(x, opname, init))


@pytest.mark.parametrize("n", [1, 33, 4097, 1 << 20, 1 << 24])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_float_scan_within_bound_and_deterministic(ex, n, dtype):
    from massively_b200 import op, vector
    x = seeded(dtype, n, seed=3)
    d = ex.to_device(x)
    got = ex.to_host(vector.inclusive_scan(ex, d, op.Add))
    exact = np.cumsum(x.astype(np.float64))
    # per-prefix bound: (i+1) * eps * sum_{k<=i} |x_k|
    eps = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
    absx = np.cumsum(np.abs(x.astype(np.float64)))
    bound = (np.arange(n) + 1) * eps * absx
    assert (np.abs(got.astype(np.float64) - exact) <= bound + 1e-30).all()
    again = ex.to_host(vector.inclusive_scan(ex, d, op.Add))
    np.testing.assert_array_equal(got.view(np.uint8), again.view(np.uint8))
    mx = ex.to_host(vector.inclusive_scan(ex, d, op.Max))
    np.testing.assert_array_equal(mx, orc.inclusive_scan(x, "max"))


def test_lazy_inputs(ex):
    from massively_b200 import lazy, op, vector
    n = 100_003
    x = seeded(np.uint32, n, 11)
    d = ex.to_device(x)
    # map(IsEven) fused into the scan load: positions of a compaction.
    got = ex.to_host(vector.inclusive_scan(ex, lazy.map(d, op.IsEven), op.Add))
    np.testing.assert_array_equal(got, np.cumsum((x & 1) == 0).astype(np.uint32))
    got = ex.to_host(vector.inclusive_scan(ex, lazy.counting(5).take(n), op.Add))
    np.testing.assert_array_equal(got, orc.inclusive_scan(np.arange(5, 5 + n, dtype=np.uint32),
                                                          "add"))
    got = ex.to_host(vector.inclusive_scan(ex, lazy.reverse(d), op.Add))
    np.testing.assert_array_equal(got, orc.inclusive_scan(x[::-1].copy(), "add"))
    idx = seeded(np.uint32, n, 12, 0, n - 1)
    got = ex.to_host(vector.inclusive_scan(ex, lazy.permute(d, ex.to_device(idx)), op.Max))
    np.testing.assert_array_equal(got, orc.inclusive_scan(x[idx], "max"))
    # u32 widened to u64 through a cast view (massively's lazy::map to u64)
    got = ex.to_host(vector.inclusive_scan(ex, lazy.cast(d, np.uint64), op.Add))
    np.testing.assert_array_equal(got, np.cumsum(x.astype(np.uint64)))


def test_unaligned_slice_and_errors(ex):
    import massively_b200 as mb
    from massively_b200 import op, vector
    x = seeded(np.uint32, 10_001, 5)
    d = ex.to_device(x)
    got = ex.to_host(vector.inclusive_scan(ex, d.slice(3, 9_000), op.Add))
    np.testing.assert_array_equal(got, orc.inclusive_scan(x[3:9000], "add"))
    other = mb.Executor(0)
    with pytest.raises(mb.ForeignExecutor):
        vector.inclusive_scan(other, d, op.Add)
    out = ex.alloc(np.uint32, 10)
    with pytest.raises(mb.OutputTooShort) as e:
        vector.inclusive_scan_into(ex, d, op.Add, out)
    assert e.value == mb.OutputTooShort(10_001, 10)
    empty = ex.to_device(np.zeros(0, np.uint32))
    assert ex.to_host(vector.inclusive_scan(ex, empty, op.Add)).size == 0


@pytest.mark.parametrize("n", [1, 8191, 8192, 8193, 100_003, 1 << 22, (1 << 24) + 5])
@pytest.mark.parametrize("dtype", [np.uint32, np.int64, np.float32, np.float64])
def test_every_scan_config(n, dtype):
    """Each scan configuration the autotuner may choose (one tile per CTA
    with a look-back warp; the same with warp 0 running the look-back; 64 KB
    tiles) gives the same results: bit-exact for integers and MAX; for float
    ADD within the bound and identical run to run."""
    from massively_b200 import op, tune, vector
    ex = executor()
    x = seeded(dtype, n, seed=n + 11)
    d = ex.to_device(x)
    for cfg in range(len(tune.configs("scan"))):
        tune.set_config(ex, "scan", cfg)
        inc = ex.to_host(vector.inclusive_scan(ex, d, op.Add))
        exc = ex.to_host(vector.exclusive_scan(ex, d, dtype(3), op.Add))
        mx = ex.to_host(vector.inclusive_scan(ex, d, op.Max))
        np.testing.assert_array_equal(mx, orc.inclusive_scan(x, "max"), err_msg=f"config {cfg}")
        if np.dtype(dtype).kind == "f":
            exact = np.cumsum(x.astype(np.float64))
            eps = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
            bound = (np.arange(n) + 1) * eps * np.cumsum(np.abs(x.astype(np.float64)))
            assert (np.abs(inc.astype(np.float64) - exact) <= bound + 1e-30).all(), cfg
            again = ex.to_host(vector.inclusive_scan(ex, d, op.Add))
            np.testing.assert_array_equal(inc.view(np.uint8), again.view(np.uint8))
        else:
            np.testing.assert_array_equal(inc, orc.inclusive_scan(x, "add"), err_msg=f"config {cfg}")
            np.testing.assert_array_equal(exc, orc.exclusive_scan(x, "add", dtype(3)),
                                          err_msg=f"config {cfg}")
    ex.sync()
