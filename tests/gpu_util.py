"""Helpers shared by the GPU parity tests (inputs, tolerances)."""
import numpy as np
import pytest

from oracle import oracle as orc


def executor():
    import massively_b200 as mb
    return mb.Executor(0)


def seeded(dtype, n, seed, lo=None, hi=None):
    """Seeded inputs from the PCG streams (massively/src/api/util/random.rs)."""
    dt = np.dtype(dtype)
    if dt == np.float32:
        return orc.normal_f32(seed, n)
    if dt == np.float64:
        return orc.normal_f32(seed, n).astype(np.float64) * 1.5
    if dt.itemsize == 8:
        lo = 0 if lo is None else lo
        hi = 0xFFFFFFFFFFFFFFFF if hi is None else hi
        return orc.uniform_u64(lo, hi, seed, n).view(dt) if dt.kind == "i" and lo == 0 and \
            hi == 0xFFFFFFFFFFFFFFFF else orc.uniform_u64(lo, hi, seed, n).astype(dt)
    lo = 0 if lo is None else lo
    hi = 0xFFFFFFFF if hi is None else hi
    u = orc.uniform_u32(lo, hi, seed, n)
    if dt.itemsize == 4:
        return u.view(dt) if dt.kind == "i" and lo == 0 and hi == 0xFFFFFFFF else u.astype(dt)
    return u.astype(dt)


def fp_bound(x, n_terms=None):
    """|err| bound of any association order of a float sum:
    n * 2^-p * sum|x| (p = 24 for f32, 53 for f64)."""
    x = np.asarray(x)
    eps = 2.0 ** -24 if x.dtype == np.float32 else 2.0 ** -53
    n = x.size if n_terms is None else n_terms
    return n * eps * float(np.abs(x.astype(np.float64)).sum())


gpu = pytest.mark.gpu
