"""Radix and comparator sort parity: CUDA path vs the oracle, bit-exact
(keys, values and stability), through the C ABI."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import known_answers as K
from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


def _perm_values(n):
    return np.arange(n, dtype=np.uint32)


def test_known_answers(ex):
    from massively_b200 import op, vector, zip3, zip7, zip12
    for case in K.RADIX:
        got = vector.radix_sort_by_key(ex, ex.to_device(case["keys"][0]),
                                       ex.to_device(case["values"]))
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    for case in K.RADIX_INTEGER_EXTREMES + K.RADIX_FLOAT_TOTAL_ORDER:
        n = case["keys"].size
        got = vector.radix_sort_by_key(ex, ex.to_device(case["keys"]),
                                       ex.to_device(_perm_values(n)))
        np.testing.assert_array_equal(ex.to_host(got), case["want"], err_msg=case["src"])
    c = K.RADIX_COMPOUND
    n = c["keys"][0].size
    vals = [np.array([col * 100 + i for i in range(n)], np.uint32) for col in range(12)]
    keys = zip3(*[ex.to_device(k) for k in c["keys"]])
    got = vector.radix_sort_by_key(ex, keys, zip7(*[ex.to_device(v) for v in vals[:7]]))
    for col, g in enumerate(got.into_columns()):
        np.testing.assert_array_equal(ex.to_host(g), vals[col][c["want"]])
    got = vector.radix_sort_by_key(ex, keys, zip12(*[ex.to_device(v) for v in vals]))
    for col, g in enumerate(got.into_columns()):
        np.testing.assert_array_equal(ex.to_host(g), vals[col][c["want"]])
    n = K.RADIX_513["n"]
    k = ((np.arange(n) * 37) % 11).astype(np.uint32)
    got = vector.radix_sort_by_key(ex, ex.to_device(k), ex.to_device(_perm_values(n)))
    np.testing.assert_array_equal(ex.to_host(got), np.argsort(k, kind="stable"))
    for case in K.SORT:
        np.testing.assert_array_equal(ex.to_host(vector.sort(ex, ex.to_device(case["x"]))),
                                      case["want"])
    for case in K.SORT_BY_KEY:
        got = vector.sort_by_key(ex, ex.to_device(case["keys"]), ex.to_device(case["values"]),
                                 op.Less)
        np.testing.assert_array_equal(ex.to_host(got), case["want"])


def test_empty_and_length_mismatch(ex):
    import massively_b200 as mb
    from massively_b200 import vector
    e = ex.to_device(np.zeros(0, np.uint32))
    assert ex.to_host(vector.radix_sort_by_key(ex, e, e)).size == 0
    with pytest.raises(mb.LengthMismatch) as err:
        vector.radix_sort_by_key(ex, ex.to_device(np.array([1, 2], np.uint32)),
                                 ex.to_device(np.array([10], np.uint32)))
    assert err.value == mb.LengthMismatch(2, 1)


SIZES = K.ORACLE_LENGTHS + [4095, 4096, 4097, 65_537, 1 << 20, 3_000_017]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("keyspace", ["full", "mod37", "16bit", "const"])
def test_u32_pairs_bit_exact(ex, n, keyspace):
    from massively_b200 import vector
    keys = seeded(np.uint32, n, seed=n + 17)
    if keyspace == "mod37":
        keys = ((np.arange(n, dtype=np.uint64) * 1103515245 + 12345) % 37).astype(np.uint32)
    elif keyspace == "16bit":
        keys = keys & np.uint32(0xFFFF)
    elif keyspace == "const":
        keys = np.full(n, 7, np.uint32)
    vals = _perm_values(n)
    sk, sv = vector.radix_sort_pairs(ex, ex.to_device(keys), ex.to_device(vals))
    want = orc.radix_perm([keys])
    np.testing.assert_array_equal(ex.to_host(sv), want)
    np.testing.assert_array_equal(ex.to_host(sk), keys[want])


@pytest.mark.parametrize("n", [0, 1, 257, 4097, 100_003, 1 << 20])
@pytest.mark.parametrize("dtype", [np.int32, np.float32, np.uint64, np.int64, np.float64])
def test_typed_keys_total_order(ex, n, dtype):
    from massively_b200 import vector
    keys = seeded(dtype, n, seed=n + 5)
    if dtype in (np.float32, np.float64) and n > 10:
        keys[: n // 50] = 0.0
        keys[n // 50: n // 25] = -0.0
        keys[-3:] = [np.inf, -np.inf, np.nan]
    vals = _perm_values(n)
    sk, sv = vector.radix_sort_pairs(ex, ex.to_device(keys), ex.to_device(vals))
    want = orc.radix_perm([keys])
    np.testing.assert_array_equal(ex.to_host(sv), want)
    np.testing.assert_array_equal(ex.to_host(sk).view(np.uint8), keys[want].view(np.uint8))
    # 64-bit payload column
    v64 = np.arange(n, dtype=np.uint64) * np.uint64(3)
    sv64 = vector.radix_sort_by_key(ex, ex.to_device(keys), ex.to_device(v64))
    np.testing.assert_array_equal(ex.to_host(sv64), v64[want])


@pytest.mark.parametrize("n", [5, 1000, 70_001])
@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.int8, np.uint16])
def test_narrow_keys(ex, n, dtype):
    from massively_b200 import vector
    keys = seeded(dtype, n, seed=9)
    got = vector.radix_sort_by_key(ex, ex.to_device(keys), ex.to_device(_perm_values(n)))
    np.testing.assert_array_equal(ex.to_host(got), orc.radix_perm([keys]))


@pytest.mark.parametrize("less", ["less", "greater", "total_less"])
@pytest.mark.parametrize("dtype", [np.uint32, np.int64, np.float32, np.float64])
def test_comparator_sorts(ex, less, dtype):
    from massively_b200 import op, vector
    n = 50_001
    keys = seeded(dtype, n, seed=21)
    if dtype in (np.float32, np.float64):
        keys[:100] = 0.0
        keys[100:200] = -0.0
        keys = keys.astype(dtype)
    else:
        keys = (keys % dtype(1000)).astype(dtype)
    o = op.pred2(less)
    got = ex.to_host(vector.sort(ex, ex.to_device(keys), o))
    want = orc.sort(keys, less)
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    vals = _perm_values(n)
    got = ex.to_host(vector.sort_by_key(ex, ex.to_device(keys), ex.to_device(vals), o))
    np.testing.assert_array_equal(got, orc.sort_perm(keys, less))


def test_lazy_keys_and_multi_values(ex):
    from massively_b200 import lazy, op, vector, zip2
    n = 100_000
    src = seeded(np.uint32, n, 33)
    d = ex.to_device(src)
    # keys = map(src, IsEven) (a lazy view) -> stable partition order
    got = vector.radix_sort_by_key(ex, lazy.map(d, op.IsEven), ex.to_device(_perm_values(n)))
    flags = ((src & 1) == 0).astype(np.uint32)
    np.testing.assert_array_equal(ex.to_host(got), np.argsort(flags, kind="stable"))
    # config-1 shape: radix_sort_by_key(keys, zip2(keys, counting))
    got = vector.radix_sort_by_key(ex, d, zip2(d, lazy.counting(0).take(n)))
    k2, v2 = got.into_columns()
    want = orc.radix_perm([src])
    np.testing.assert_array_equal(ex.to_host(k2), src[want])
    np.testing.assert_array_equal(ex.to_host(v2), want)


def test_large_pairs(ex):
    from massively_b200 import vector
    n = 1 << 24
    keys = seeded(np.uint32, n, 0)
    vals = _perm_values(n)
    sk, sv = vector.radix_sort_pairs(ex, ex.to_device(keys), ex.to_device(vals))
    want = np.argsort(keys, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(ex.to_host(sv), want)
    np.testing.assert_array_equal(ex.to_host(sk), keys[want])


@pytest.mark.parametrize("n", [1, 4095, 4096, 65_537, 1 << 20])
@pytest.mark.parametrize("keyspace", ["full", "16bit", "const"])
def test_every_radix_config_bit_exact(n, keyspace):
    """Each onesweep configuration the autotuner may choose sorts the same."""
    from massively_b200 import tune, vector
    ex = executor()
    keys = seeded(np.uint32, n, seed=n + 5)
    if keyspace == "16bit":
        keys = keys & np.uint32(0xFFFF)
    elif keyspace == "const":
        keys = np.full(n, 3, np.uint32)
    vals = _perm_values(n)
    want = orc.radix_perm([keys])
    for cfg in range(len(tune.configs("radix"))):
        tune.set_config(ex, "radix", cfg)
        for kdt in (np.uint32, np.float32):
            k = keys.view(kdt)
            sk, sv = vector.radix_sort_pairs(ex, ex.to_device(k), ex.to_device(vals))
            w = want if kdt == np.uint32 else orc.radix_perm([k])
            np.testing.assert_array_equal(ex.to_host(sv), w, err_msg=f"config {cfg} {kdt}")
    ex.sync()


def test_kernel_timing_counts_onesweep_launches():
    """mb_kernel_timing brackets each onesweep pass and the histogram."""
    import ctypes as C
    from massively_b200 import _native as N, vector
    ex = executor()
    L = N.lib()
    n = 1 << 20
    keys, vals = ex.to_device(seeded(np.uint32, n, 9)), ex.to_device(_perm_values(n))
    for fam in range(4):
        L.mb_kernel_timing_read(ex.handle, fam, None, None)
    L.mb_kernel_timing(ex.handle, 1)
    vector.radix_sort_pairs(ex, keys, vals)
    vector.radix_sort_pairs(ex, keys, vals)
    L.mb_kernel_timing(ex.handle, 0)
    vector.radix_sort_pairs(ex, keys, vals)  # not recorded
    got = {}
    for fam in (N.KF_RADIX_ONESWEEP, N.KF_RADIX_HISTOGRAM, N.KF_SCAN):
        cnt, ms = C.c_uint64(), C.c_double()
        assert L.mb_kernel_timing_read(ex.handle, fam, C.byref(cnt), C.byref(ms)) == 0
        got[fam] = (cnt.value, ms.value)
    assert got[N.KF_RADIX_ONESWEEP][0] == 8 and got[N.KF_RADIX_ONESWEEP][1] > 0
    assert got[N.KF_RADIX_HISTOGRAM][0] == 2
    assert got[N.KF_SCAN] == (0, 0.0)
    cnt = C.c_uint64()
    L.mb_kernel_timing_read(ex.handle, N.KF_RADIX_ONESWEEP, C.byref(cnt), None)
    assert cnt.value == 0  # read forgets


def test_autotune_records_and_selects_fastest(tmp_path):
    """autotune times every radix shape on the caller's workload, persists
    the fastest for (device, family, dtype, size bucket) and selects it; the
    sort stays bit-exact under the chosen shape."""
    import torch

    from massively_b200 import _native as N, tune, vector
    ex = executor()
    n = 1 << 20
    keys = seeded(np.uint32, n, 21)
    vals = _perm_values(n)
    dk, dv = ex.to_device(keys), ex.to_device(vals)
    db = str(tmp_path / "tune.json")
    best = tune.autotune(ex, "radix", "u32", n, lambda: vector.radix_sort_pairs(ex, dk, dv),
                         reps=2, warmup=1, path=db)
    assert 0 <= best < len(tune.configs("radix"))
    assert N.lib().mb_tune_get(ex.handle, tune.FAMILIES["radix"]) == best
    assert tune.lookup(torch.cuda.get_device_name(0), "radix", "u32", n, db) == best
    sk, sv = vector.radix_sort_pairs(ex, dk, dv)
    np.testing.assert_array_equal(ex.to_host(sv), orc.radix_perm([keys]))
    tune.set_config(ex, "radix", -1)
    ex.sync()


def test_radix_sort_beyond_2e30_items(ex):
    """massively's length contract is any length that fits u32
    (massively/src/lib.rs:82, core/runtime.rs:14-19): 2^30 + 5 (u32 key,
    u32 value = index) pairs, with 60% of the keys sharing their second byte
    (one digit bucket then holds more than 2^29 items).  The result is the
    unique stable order: output keys are the input keys at the output
    values, (key, value) strictly increases (sorted, and stable since the
    values are the input positions), and the values are a permutation."""
    import torch

    import bench
    from massively_b200 import lazy, vector
    n = (1 << 30) + 5
    kd = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 21, n)
    sel = bench.device_uniform_u32(ex, 0, 0xFFFFFFFF, 22, n)
    k64 = kd.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    skew = (sel.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF) < int(0.6 * 2 ** 32)
    k64 = torch.where(skew, (k64 & ~0xFF00) | 0x5A00, k64)
    kd.tensor.view(torch.int32).copy_(k64.to(torch.int32))
    del sel, skew, k64
    vd = ex.alloc(np.uint32, n)
    vector.copy(ex, lazy.counting(0).take(n), vd)
    sk, sv = vector.radix_sort_pairs(ex, kd, vd)
    ex.sync()
    del vd
    torch.cuda.empty_cache()
    k = sk.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    v = sv.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    del sk, sv
    kin = kd.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    assert torch.equal(kin[v], k), "output keys are not the input keys at the output values"
    del kin
    comp = k * (1 << 31) + v  # below 2^63: k < 2^32, v < 2^31
    assert bool((comp[1:] > comp[:-1]).all()), "not sorted and stable"
    del comp, k
    seen = torch.zeros(n, dtype=torch.int8, device=v.device)
    seen[v] = 1
    assert bool(seen.all()), "values are not a permutation"
