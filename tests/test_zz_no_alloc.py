"""The allocation-free inclusive scan (mb_inclusive_scan_noalloc).

Some callers may not allocate device memory in the middle of their work --
for example code running while another allocator has reserved all free
device memory, or code that must never meet an allocation failure or an
allocator synchronisation partway through.  For them the library exports a
scan whose look-back scratch is a fixed array in the library's device
memory.  These tests call it through the C ABI and check it against the
regular mb_inclusive_scan on the same inputs (bit-exact: integer results,
and for floats the same fixed association) and, for narrow, lazy and
device-length inputs, against the CPU oracle directly -- each twice in a row
so a second call cannot see stale scratch from the first.  This file sorts
last so a run that stops at the first failure has already run every other
test.
"""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_util import gpu, seeded

pytestmark = gpu


def _scan(ex, fn_name, x_dev, op_id, out):
    from massively_b200 import _native as N
    from massively_b200.runtime import check
    s = x_dev.to_src()
    check(getattr(N.lib(), fn_name)(ex.handle, C.byref(s), op_id, out.to_col()))


@pytest.mark.parametrize("dtype,n", [(np.uint32, 1_000_003), (np.uint32, 1 << 22),
                                     (np.float32, 1 << 20), (np.uint64, 300_001),
                                     (np.int32, 4097)])
def test_noalloc_scan_matches_regular_scan_twice(dtype, n):
    import massively_b200 as mb
    from massively_b200 import op
    ex = mb.Executor(0)
    for call in range(2):  # two calls in a row; the second must not see stale state
        x = seeded(dtype, n, seed=17 + call)
        d = ex.to_device(x)
        want = ex.alloc(dtype, n)
        got = ex.alloc(dtype, n)
        _scan(ex, "mb_inclusive_scan", d, op.Add.id, want)
        _scan(ex, "mb_inclusive_scan_noalloc", d, op.Add.id, got)
        ex.sync()
        np.testing.assert_array_equal(ex.to_host(got).view(np.uint8),
                                      ex.to_host(want).view(np.uint8))
        _scan(ex, "mb_inclusive_scan_noalloc", d, op.Max.id, got)
        _scan(ex, "mb_inclusive_scan", d, op.Max.id, want)
        ex.sync()
        np.testing.assert_array_equal(ex.to_host(got).view(np.uint8),
                                      ex.to_host(want).view(np.uint8))


def _scan_src(ex, src, op_id, out):
    from massively_b200 import _native as N
    from massively_b200.runtime import check
    check(N.lib().mb_inclusive_scan_noalloc(ex.handle, C.byref(src), op_id, out.to_col()))


def test_noalloc_scan_narrow_and_lazy_inputs_match_oracle_twice(orc):
    """The register-tiled kernel (an int8 column, and a lazy cast view of it)
    against the CPU oracle directly, twice in a row."""
    import massively_b200 as mb
    from massively_b200 import lazy, op
    ex = mb.Executor(0)
    n = 300_007
    for call in range(2):
        x = seeded(np.int8, n, seed=31 + call)
        d = ex.to_device(x)
        got8 = ex.alloc(np.int8, n)
        _scan_src(ex, d.to_src(), op.Add.id, got8)
        keep = []
        src = lazy.lower(ex, lazy.cast(d, np.int32), keep)
        got32 = ex.alloc(np.int32, n)
        _scan_src(ex, src, op.Add.id, got32)
        ex.sync()
        np.testing.assert_array_equal(ex.to_host(got8), orc.inclusive_scan(x, "add"))
        np.testing.assert_array_equal(ex.to_host(got32),
                                      orc.inclusive_scan(x.astype(np.int32), "add"))


def test_noalloc_scan_device_length_matches_oracle_twice(orc):
    """A column whose logical length is a count on the device: only that
    many items are scanned and written."""
    import massively_b200 as mb
    from massively_b200 import op
    ex = mb.Executor(0)
    n = 1 << 20
    for call, m in enumerate([n // 3 + 7, 4097]):
        x = seeded(np.uint32, n, seed=41 + call)
        cnt = ex.to_device(np.array([m], np.uint32))
        d = ex.to_device(x).with_len_dev(cnt.tensor)
        got = ex.zeros(np.uint32, n)
        _scan_src(ex, d.to_src(), op.Add.id, got)
        ex.sync()
        h = ex.to_host(got)
        np.testing.assert_array_equal(h[:m], orc.inclusive_scan(x[:m], "add"))
        assert not h[m:].any()


def test_noalloc_scan_rejects_sizes_beyond_its_limit():
    import massively_b200 as mb
    from massively_b200 import _native as N
    from massively_b200 import op
    ex = mb.Executor(0)
    big = ex.alloc(np.uint64, (1 << 26) + 1)
    out = ex.alloc(np.uint64, (1 << 26) + 1)
    s = big.to_src()
    rc = N.lib().mb_inclusive_scan_noalloc(ex.handle, C.byref(s), op.Add.id, out.to_col())
    assert rc == N.LENGTH_TOO_LARGE
    assert b"allocation-free scan" in N.lib().mb_last_error_message()
