"""User operators compile on the host (NVRTC needs no device): a valid
operator compiles for sm_100a, a broken one is reported as a launch error
carrying the compiler's message."""
import numpy as np
import pytest


def _nvrtc_available():
    import ctypes
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            ctypes.CDLL(name)
            return True
        except OSError:
            continue
    return False


pytestmark = pytest.mark.skipif(not _nvrtc_available(), reason="NVRTC not installed")


def test_binary_and_map_sources_compile():
    from massively_b200.op import UserOp
    UserOp.check_source(0, np.uint32, np.uint32,
                        "__device__ T sat_add(T a, T b) { T s = a + b; return s < a ? ~0u : s; }",
                        "sat_add")
    UserOp.check_source(1, np.float32, np.int32,
                        "__device__ Out bucket(In x) { return (Out)(x * 4.0f); }", "bucket")


def test_compile_error_is_reported():
    from massively_b200.op import UserOp
    from massively_b200.runtime import Error
    with pytest.raises(Error) as e:
        UserOp.check_source(0, np.uint32, np.uint32, "__device__ T broken(T a, T b) { return a +; }",
                            "broken")
    assert "did not compile" in str(e.value)


def test_comparator_sources_compile():
    """A user comparator (kind 2) compiles with the merge-sort kernels; a
    broken one reports the compiler's message."""
    from massively_b200.op import UserOp
    from massively_b200.runtime import Error
    for dt in (np.uint32, np.float64, np.int16):
        UserOp.check_source(2, dt, dt, "__device__ bool by_low(T a, T b) { return (a & 7) < (b & 7); }"
                            if np.dtype(dt).kind in "iu" else
                            "__device__ bool desc(T a, T b) { return b < a; }",
                            "by_low" if np.dtype(dt).kind in "iu" else "desc")
    with pytest.raises(Error) as e:
        UserOp.check_source(2, np.uint32, np.uint32, "__device__ bool bad(T a, T b) { return a <; }",
                            "bad")
    assert "did not compile" in str(e.value)
