"""numpy front end of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg; the product package never
imports it.  Every function restates one function of massively's CPU
reference (verification/oracle/src/vector.rs, verification/oracle/src/seg.rs)
and cites it; the C++ side holds the loops.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

# mb_dtype / mb_op / mb_pred2 / mb_unary ids (include/massively_b200.h)
DTYPES = {
    np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.uint32): 2,
    np.dtype(np.uint64): 3, np.dtype(np.int8): 4, np.dtype(np.int16): 5,
    np.dtype(np.int32): 6, np.dtype(np.int64): 7, np.dtype(np.float32): 8,
    np.dtype(np.float64): 9,
}
OPS = {"add": 0, "mul": 1, "min": 2, "max": 3, "and": 4, "or": 5, "xor": 6,
       "take_left": 7, "take_right": 8}
PRED2 = {"less": 0, "greater": 1, "total_less": 2, "equal": 3}
UNARY = {"identity": 0, "is_true": 1, "is_false": 2, "is_even": 3, "is_odd": 4,
         "negate": 5, "bit_not": 6, "abs": 7, "is_negative": 8, "is_positive": 9}

_lib = None


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    vp, u64, i32, i64, u32 = C.c_void_p, C.c_uint64, C.c_int, C.c_int64, C.c_uint32
    sig = {
        "orc_pcg_hash32": (u32, [u32]),
        "orc_seed_key": (u32, [u64]),
        "orc_uniform_u32": (None, [u32, u32, u64, u64, u64, vp]),
        "orc_uniform_u64": (None, [u64, u64, u64, u64, u64, vp]),
        "orc_normal_f32": (None, [u64, u64, u64, vp]),
        "orc_reduce": (i32, [i32, vp, u64, i32, vp, vp]),
        "orc_inclusive_scan": (i32, [i32, vp, u64, i32, vp]),
        "orc_exclusive_scan": (i32, [i32, vp, u64, i32, vp, vp]),
        "orc_copy_where": (i64, [vp, u64, u64, vp, vp]),
        "orc_remove_where": (i64, [vp, u64, u64, vp, vp]),
        "orc_partition": (i64, [i32, vp, u64, i32, vp]),
        "orc_gather": (None, [vp, u64, vp, vp, u64, vp]),
        "orc_scatter": (None, [vp, u64, vp, vp, u64, vp]),
        "orc_replace_where": (None, [vp, u64, vp, u64, vp]),
        "orc_masked_copy": (None, [vp, u64, vp, u64, vp]),
        "orc_sort_perm": (i32, [i32, vp, u64, i32, vp]),
        "orc_radix_perm": (i32, [i32, vp, vp, u64, vp]),
        "orc_radix_perm_par": (i32, [i32, vp, u64, i32, vp]),
        "orc_run_heads": (i32, [i32, vp, u64, i32, vp]),
        "orc_adjacent_heads": (i32, [i32, vp, u64, i32, vp]),
        "orc_runs_reduce": (i64, [i32, vp, u64, vp, i32, vp, vp]),
        "orc_reduce_by_key_u32": (i64, [vp, vp, u64, i32, u32, vp, vp]),
        "orc_scan_by_key": (i32, [i32, vp, u64, vp, i32, i32, vp, vp]),
        "orc_merge_src": (i32, [i32, vp, u64, vp, u64, i32, vp]),
        "orc_bounds": (i32, [i32, vp, u64, vp, u64, i32, i32, vp]),
        "orc_set_op_src": (i64, [i32, vp, u64, vp, u64, i32, i32, vp]),
        "orc_unique": (i64, [i32, vp, u64, i32, vp]),
        "orc_find": (i64, [i32, i32, vp, u64, vp, u64, i32]),
        "orc_scatter_reduce": (i32, [i32, vp, vp, u64, i32, vp, vp, u64]),
        "orc_seg_query": (i32, [i32, vp, vp, u64, i32, i32, vp]),
        "orc_seg_transform": (i64, [i32, vp, vp, u64, i32, i32, vp, vp]),
        "orc_arg": (i32, [i32, i32, vp, u64, i32, vp]),
        "orc_seg_scan": (i32, [i32, vp, vp, u64, i32, i32, vp, vp]),
        "orc_seg_reduce": (i32, [i32, vp, vp, u64, i32, vp, vp]),
        "orc_seg_sort": (i32, [i32, vp, vp, u64, i32, vp]),
        "orc_validate_offsets": (i64, [vp, u64]),
        "orc_scale_lcg": (None, [u64, vp]),
        "orc_scale_other": (None, [u64, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a)


def _dt(a: np.ndarray) -> int:
    return DTYPES[a.dtype]


def _scalar(value, dtype) -> np.ndarray:
    return np.array([value], dtype=dtype)


# ------------------------------------------------------------------ random --

def pcg_hash32(x: int) -> int:
    """random.rs:12-16."""
    return int(lib().orc_pcg_hash32(x & 0xFFFFFFFF))


def seed_key(seed: int) -> int:
    """random.rs:18-22."""
    return int(lib().orc_seed_key(seed))


def uniform_u32(lo: int, hi: int, seed: int, n: int, offset: int = 0) -> np.ndarray:
    """util::random::uniform_u32(lo, hi, seed).take(n) (random.rs:376-385)."""
    out = np.empty(n, np.uint32)
    lib().orc_uniform_u32(lo, hi, seed, offset, n, _p(out))
    return out


def uniform_u64(lo: int, hi: int, seed: int, n: int, offset: int = 0) -> np.ndarray:
    """util::random::uniform_u64 (random.rs:343-348, 387-396)."""
    out = np.empty(n, np.uint64)
    lib().orc_uniform_u64(lo, hi, seed, offset, n, _p(out))
    return out


def normal_f32(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Host f64 Box-Muller N(0,1) on the PCG streams, rounded to f32."""
    out = np.empty(n, np.float32)
    lib().orc_normal_f32(seed, offset, n, _p(out))
    return out


def scale_input(n: int) -> np.ndarray:
    """vector_scale/common.rs:138-142 LCG."""
    out = np.empty(n, np.uint32)
    lib().orc_scale_lcg(n, _p(out))
    return out


def scale_other(n: int) -> np.ndarray:
    """vector_scale/common.rs:144-148 LCG."""
    out = np.empty(n, np.uint32)
    lib().orc_scale_other(n, _p(out))
    return out


# ------------------------------------------------------------------ vector --

def reduce(x, op: str, init):
    """vector.rs:33-42: init op x0 op x1 ... (left fold)."""
    x = _c(x)
    i = _scalar(init, x.dtype)
    o = np.empty(1, x.dtype)
    lib().orc_reduce(_dt(x), _p(x), x.size, OPS[op], _p(i), _p(o))
    return o[0]


def inclusive_scan(x, op: str) -> np.ndarray:
    """vector.rs:44-59."""
    x = _c(x)
    o = np.empty_like(x)
    lib().orc_inclusive_scan(_dt(x), _p(x), x.size, OPS[op], _p(o))
    return o


def exclusive_scan(x, op: str, init) -> np.ndarray:
    """vector.rs:61-74."""
    x = _c(x)
    i = _scalar(init, x.dtype)
    o = np.empty_like(x)
    lib().orc_exclusive_scan(_dt(x), _p(x), x.size, OPS[op], _p(i), _p(o))
    return o


def _rows(cols):
    cols = [_c(c) for c in cols]
    n = cols[0].size
    rec = np.empty(n, dtype=[(f"c{k}", c.dtype) for k, c in enumerate(cols)])
    for k, c in enumerate(cols):
        rec[f"c{k}"] = c
    return rec


def _unrows(rec, k):
    return [np.ascontiguousarray(rec[f"c{j}"]) for j in range(k)]


def copy_where(cols, stencil):
    """vector.rs:255-262: rows whose flag is non-zero, in order."""
    single = isinstance(cols, np.ndarray)
    cols = [cols] if single else list(cols)
    rec = _rows(cols)
    st = _c(np.asarray(stencil, np.uint32))
    out = np.empty_like(rec)
    k = lib().orc_copy_where(_p(rec), rec.size, rec.dtype.itemsize, _p(st), _p(out))
    res = _unrows(out[:k], len(cols))
    return res[0] if single else res


def remove_where(cols, stencil):
    """vector.rs:264-271."""
    single = isinstance(cols, np.ndarray)
    cols = [cols] if single else list(cols)
    rec = _rows(cols)
    st = _c(np.asarray(stencil, np.uint32))
    out = np.empty_like(rec)
    k = lib().orc_remove_where(_p(rec), rec.size, rec.dtype.itemsize, _p(st), _p(out))
    res = _unrows(out[:k], len(cols))
    return res[0] if single else res


def partition(x, pred: str):
    """vector.rs:216-233: (matching ++ failing, boundary)."""
    x = _c(x)
    o = np.empty_like(x)
    b = lib().orc_partition(_dt(x), _p(x), x.size, UNARY[pred], _p(o))
    return o, int(b)


def flags(x, pred: str) -> np.ndarray:
    """Element-wise predicate -> MFlag (the lazy::map(x, Pred) stencil)."""
    x = np.asarray(x)
    if pred == "is_true":
        return (x != 0).astype(np.uint32)
    if pred == "is_false":
        return (x == 0).astype(np.uint32)
    if pred == "is_even":
        return ((x.astype(np.uint64) & 1) == 0).astype(np.uint32)
    if pred == "is_odd":
        return ((x.astype(np.uint64) & 1) != 0).astype(np.uint32)
    if pred == "is_negative":
        return (x < 0).astype(np.uint32)
    if pred == "is_positive":
        return (x > 0).astype(np.uint32)
    raise ValueError(pred)


def gather(src, idx, stencil=None, out=None):
    """vector.rs:285-297."""
    src = _c(src)
    idx = _c(np.asarray(idx, np.uint32))
    out = np.zeros(idx.size, src.dtype) if out is None else _c(out.copy())
    st = None if stencil is None else _c(np.asarray(stencil, np.uint32))
    lib().orc_gather(_p(src), src.itemsize, _p(idx), None if st is None else _p(st), idx.size,
                     _p(out))
    return out


def scatter(src, idx, out, stencil=None):
    """vector.rs:299-311."""
    src = _c(src)
    idx = _c(np.asarray(idx, np.uint32))
    out = _c(np.array(out, copy=True))
    st = None if stencil is None else _c(np.asarray(stencil, np.uint32))
    lib().orc_scatter(_p(src), src.itemsize, _p(idx), None if st is None else _p(st), src.size,
                      _p(out))
    return out


def replace_where(value, stencil, out):
    """vector.rs:277-283: a new array, `value` where stencil[i] != 0."""
    o = _c(np.array(out, copy=True))
    st = _c(np.asarray(stencil, np.uint32))
    v = _scalar(value, o.dtype)
    lib().orc_replace_where(_p(v), o.itemsize, _p(st), o.size, _p(o))
    return o


def transform_where(source, op, stencil, out):
    """vector.rs:20-31: a new array, op(source[i]) where stencil[i] != 0;
    `op` is a host function mapping an array to its results (the operator
    applied item by item)."""
    o = _c(np.array(out, copy=True))
    res = _c(np.asarray(op(np.asarray(source)), dtype=o.dtype))
    st = _c(np.asarray(stencil, np.uint32))
    lib().orc_masked_copy(_p(res), o.itemsize, _p(st), o.size, _p(o))
    return o


def sort_perm(keys, less: str = "less") -> np.ndarray:
    """Stable comparator order (vector.rs:483-491, 666-680)."""
    keys = _c(keys)
    perm = np.empty(keys.size, np.uint32)
    lib().orc_sort_perm(_dt(keys), _p(keys), keys.size, PRED2[less], _p(perm))
    return perm


def sort(keys, less: str = "less") -> np.ndarray:
    """vector.rs:483-491."""
    keys = _c(keys)
    return keys[sort_perm(keys, less)]


def sort_by_key(keys, values, less: str = "less"):
    """vector.rs:515-524; `values` may be one array or a list of columns."""
    keys = _c(keys)
    perm = sort_perm(keys, less)
    if isinstance(values, np.ndarray):
        return keys[perm], _c(values)[perm]
    return keys[perm], [_c(v)[perm] for v in values]


def radix_perm(key_cols) -> np.ndarray:
    """Stable order of up to three key columns in radix total order
    (massively/src/core/radix.rs:46-89, 500-531)."""
    key_cols = [_c(k) for k in key_cols]
    n = key_cols[0].size
    dts = np.array([_dt(k) for k in key_cols], np.int32)
    ptrs = (C.c_void_p * len(key_cols))(*[k.ctypes.data for k in key_cols])
    perm = np.empty(n, np.uint32)
    lib().orc_radix_perm(len(key_cols), _p(dts), C.cast(ptrs, C.c_void_p), n, _p(perm))
    return perm


def radix_perm_par(keys, threads: int | None = None) -> np.ndarray:
    """radix_perm of one key column on several host threads, for full
    benchmark sizes: the same permutation (a stable order is the order by
    (encoded key, input index), which the threads sort and merge)."""
    import os
    keys = _c(keys)
    perm = np.empty(keys.size, np.uint32)
    rc = lib().orc_radix_perm_par(_dt(keys), _p(keys), keys.size,
                                  int(threads or os.cpu_count() or 1), _p(perm))
    if rc != 0:
        raise ValueError("radix_perm_par takes one 32- or 64-bit key column below 2^32 items")
    return perm


def radix_sort_by_key(key_cols, val_cols):
    """vector::radix_sort_by_key: the value columns permuted into radix order."""
    if isinstance(key_cols, np.ndarray):
        key_cols = [key_cols]
    single = isinstance(val_cols, np.ndarray)
    vals = [val_cols] if single else list(val_cols)
    perm = radix_perm(key_cols)
    res = [_c(v)[perm] for v in vals]
    return res[0] if single else res


def run_heads(keys, key_eq: str = "equal") -> np.ndarray:
    """Run heads of reduce_by_key (vector.rs:144-174: compare with the head)."""
    keys = _c(keys)
    h = np.empty(keys.size, np.uint8)
    lib().orc_run_heads(_dt(keys), _p(keys), keys.size, PRED2[key_eq], _p(h))
    return h


def reduce_by_key(keys, values, ops, inits, key_eq: str = "equal"):
    """vector.rs:144-174 with one or more value columns sharing the runs.

    Returns (unique_keys, [reduced column per value column])."""
    keys = _c(keys)
    single = isinstance(values, np.ndarray)
    vals = [values] if single else list(values)
    ops = [ops] * len(vals) if isinstance(ops, str) else list(ops)
    inits = [inits] * len(vals) if np.isscalar(inits) else list(inits)
    h = run_heads(keys, key_eq)
    out_keys = keys[h.astype(bool)]
    outs = []
    for v, op, init in zip(vals, ops, inits):
        v = _c(v)
        o = np.empty(max(1, v.size), v.dtype)
        i = _scalar(init, v.dtype)
        r = lib().orc_runs_reduce(_dt(v), _p(v), v.size, _p(h), OPS[op], _p(i), _p(o))
        outs.append(o[:r])
    return out_keys, (outs[0] if single else outs)


def reduce_by_key_literal_u32(keys, values, op: str, init: int):
    """The loop of vector.rs:144-174 verbatim, for u32 keys / values."""
    keys = _c(np.asarray(keys, np.uint32))
    values = _c(np.asarray(values, np.uint32))
    ok = np.empty(max(1, keys.size), np.uint32)
    ov = np.empty(max(1, keys.size), np.uint32)
    r = lib().orc_reduce_by_key_u32(_p(keys), _p(values), keys.size, OPS[op], init, _p(ok),
                                    _p(ov))
    return ok[:r], ov[:r]


def scan_by_key(keys, values, op: str, exclusive: bool = False, init=0,
                key_eq: str = "equal") -> np.ndarray:
    """vector.rs:92-142 (segments split where adjacent keys differ)."""
    keys = _c(keys)
    values = _c(values)
    h = np.empty(keys.size, np.uint8)
    lib().orc_adjacent_heads(_dt(keys), _p(keys), keys.size, PRED2[key_eq], _p(h))
    o = np.empty_like(values)
    i = _scalar(init, values.dtype)
    lib().orc_scan_by_key(_dt(values), _p(values), values.size, _p(h), OPS[op], int(exclusive),
                          _p(i), _p(o))
    return o


def _apply_src(src, left_cols, right_cols):
    right = (src >> np.uint64(63)).astype(bool)
    idx = (src & np.uint64((1 << 63) - 1)).astype(np.int64)
    outs = []
    for lc, rc in zip(left_cols, right_cols):
        lc, rc = _c(lc), _c(rc)
        o = np.empty(src.size, lc.dtype)
        o[~right] = lc[idx[~right]]
        o[right] = rc[idx[right]]
        outs.append(o)
    return outs


def merge(left, right, less: str = "less") -> np.ndarray:
    """vector.rs:493-513."""
    left, right = _c(left), _c(right)
    src = np.empty(left.size + right.size, np.uint64)
    lib().orc_merge_src(_dt(left), _p(left), left.size, _p(right), right.size, PRED2[less],
                        _p(src))
    return _apply_src(src, [left], [right])[0]


def lower_bound(source, values, less: str = "less") -> np.ndarray:
    """vector.rs:404-414: first index whose candidate is not less than each value."""
    source, values = _c(source), _c(values)
    out = np.empty(values.size, np.uint32)
    lib().orc_bounds(_dt(source), _p(source), source.size, _p(values), values.size, PRED2[less],
                     0, _p(out))
    return out


def upper_bound(source, values, less: str = "less") -> np.ndarray:
    """vector.rs:416-426: first index whose candidate each value is less than."""
    source, values = _c(source), _c(values)
    out = np.empty(values.size, np.uint32)
    lib().orc_bounds(_dt(source), _p(source), source.size, _p(values), values.size, PRED2[less],
                     1, _p(out))
    return out


def merge_by_key(lk, lv, rk, rv, less: str = "less"):
    """vector.rs:526-558."""
    lk, rk = _c(lk), _c(rk)
    src = np.empty(lk.size + rk.size, np.uint64)
    lib().orc_merge_src(_dt(lk), _p(lk), lk.size, _p(rk), rk.size, PRED2[less], _p(src))
    single = isinstance(lv, np.ndarray)
    lvs = [lv] if single else list(lv)
    rvs = [rv] if single else list(rv)
    keys = _apply_src(src, [lk], [rk])[0]
    vals = _apply_src(src, lvs, rvs)
    return keys, (vals[0] if single else vals)


def _set_op(left, right, less, mode):
    left, right = _c(left), _c(right)
    src = np.empty(left.size + right.size, np.uint64)
    k = lib().orc_set_op_src(_dt(left), _p(left), left.size, _p(right), right.size,
                             PRED2[less], mode, _p(src))
    return _apply_src(src[:k], [left], [right])[0]


def set_union(left, right, less: str = "less") -> np.ndarray:
    """vector.rs:595-619."""
    return _set_op(left, right, less, 0)


def set_intersection(left, right, less: str = "less") -> np.ndarray:
    """vector.rs:621-642."""
    return _set_op(left, right, less, 1)


def set_difference(left, right, less: str = "less") -> np.ndarray:
    """vector.rs:644-664."""
    return _set_op(left, right, less, 2)


def unique(x, eq: str = "equal") -> np.ndarray:
    """vector.rs:560-576."""
    x = _c(x)
    o = np.empty_like(x)
    k = lib().orc_unique(_dt(x), _p(x), x.size, PRED2[eq], _p(o))
    return o[:k]


# --------------------------------------------------------------------- seg --

def scatter_reduce(values, indices, init, op: str, out):
    """massively/src/api/algorithm/scatter.rs:332-420: out[d] op (init op
    v ...) per destination, proposals in input order; returns a new array."""
    values, indices = _c(values), _c(indices).astype(np.uint32)
    o = np.array(out, copy=True)
    if o.dtype != values.dtype:
        raise TypeError("output element type differs from the values'")
    iv = _scalar(init, values.dtype)
    if lib().orc_scatter_reduce(_dt(values), _p(values), _p(indices), values.size, OPS[op],
                                _p(iv), _p(o), o.size) != 0:
        raise TypeError(values.dtype)
    return o


NONE = 0xFFFFFFFF  # MIndex::MAX, massively's None


def _find(kind: int, a, b=None, op: int = 0):
    a = _c(a)
    b = a if b is None else _c(b)
    if a.dtype != b.dtype:
        raise TypeError("element types differ")
    r = lib().orc_find(kind, _dt(a), _p(a), a.size, _p(b), b.size, op)
    if r < 0:
        raise TypeError(a.dtype)
    return int(r)


def _opt(r: int):
    return None if r == NONE else r


def count_if(x, pred: str) -> int:
    """vector.rs:176-186."""
    return int(flags(x, pred).sum())


def all_of(x, pred: str) -> bool:
    """vector.rs:188-194."""
    return bool(flags(x, pred).all())


def any_of(x, pred: str) -> bool:
    """vector.rs:196-202."""
    return bool(flags(x, pred).any())


def none_of(x, pred: str) -> bool:
    """vector.rs:204-210."""
    return not any_of(x, pred)


def find_if(x, pred: str):
    """vector.rs:212-218: first passing position, or None."""
    return _opt(_find(0, x, op=UNARY[pred]))


def is_partitioned(x, pred: str) -> bool:
    """massively/src/core/predicate.rs:111-127, 213-223: no passing item
    follows a failing one."""
    return bool(_find(1, x, op=UNARY[pred]))


def adjacent_find(x, eq: str = "equal"):
    """vector.rs:344-352."""
    return _opt(_find(2, x))


def is_sorted_until(x, less: str = "less") -> int:
    """vector.rs:367-377."""
    return _find(3, x, op=PRED2[less])


def is_sorted(x, less: str = "less") -> bool:
    """vector.rs:379-386."""
    return is_sorted_until(x, less) == np.asarray(x).size


def mismatch(left, right, eq: str = "equal"):
    """vector.rs:330-342."""
    return _opt(_find(4, left, right))


def equal(left, right, eq: str = "equal") -> bool:
    """vector.rs:317-328."""
    return bool(_find(5, left, right))


def lexicographical_compare(left, right, less: str = "less") -> bool:
    """vector.rs:388-402."""
    return bool(_find(6, left, right, PRED2[less]))


def find_first_of(source, needles, eq: str = "equal"):
    """vector.rs:354-365."""
    return _opt(_find(7, source, needles))


def _arg(kind: int, x, less: str):
    x = _c(x)
    out = np.zeros(2, np.uint32)
    if lib().orc_arg(kind, _dt(x), _p(x), x.size, PRED2[less], _p(out)) != 0:
        raise TypeError(x.dtype)
    return out


def min_element(x, less: str = "less"):
    """vector.rs:428-443: first minimum, or None."""
    return _opt(int(_arg(0, x, less)[0]))


def max_element(x, less: str = "less"):
    """vector.rs:445-460: first maximum, or None."""
    return _opt(int(_arg(1, x, less)[0]))


def minmax_element(x, less: str = "less"):
    """vector.rs:462-481: (last minimum, first maximum), or None."""
    o = _arg(2, x, less)
    return None if o[0] == NONE else (int(o[0]), int(o[1]))


def validate_offsets(offsets):
    """Segmentation::from_offsets rules; value count, or None if invalid."""
    off = _c(np.asarray(offsets, np.uint32))
    r = lib().orc_validate_offsets(_p(off), off.size)
    return None if r < 0 else int(r)


def seg_inclusive_scan(x, offsets, op: str) -> np.ndarray:
    """seg.rs:48-68."""
    x = _c(x)
    off = _c(np.asarray(offsets, np.uint32))
    o = np.empty_like(x)
    z = np.zeros(1, x.dtype)
    lib().orc_seg_scan(_dt(x), _p(x), _p(off), off.size - 1, OPS[op], 0, _p(z), _p(o))
    return o


def seg_exclusive_scan(x, offsets, op: str, init) -> np.ndarray:
    """seg.rs:70-88."""
    x = _c(x)
    off = _c(np.asarray(offsets, np.uint32))
    o = np.empty_like(x)
    i = _scalar(init, x.dtype)
    lib().orc_seg_scan(_dt(x), _p(x), _p(off), off.size - 1, OPS[op], 1, _p(i), _p(o))
    return o


def seg_reduce(x, offsets, op: str, init) -> np.ndarray:
    """seg.rs:155-169."""
    x = _c(x)
    off = _c(np.asarray(offsets, np.uint32))
    o = np.empty(off.size - 1, x.dtype)
    i = _scalar(init, x.dtype)
    lib().orc_seg_reduce(_dt(x), _p(x), _p(off), off.size - 1, OPS[op], _p(i), _p(o))
    return o


def seg_sort(x, offsets, less: str = "less") -> np.ndarray:
    """seg.rs:18-39."""
    x = _c(x)
    off = _c(np.asarray(offsets, np.uint32))
    o = np.empty_like(x)
    lib().orc_seg_sort(_dt(x), _p(x), _p(off), off.size - 1, PRED2[less], _p(o))
    return o


SEG_QUERIES = {"count_if": 0, "find_if": 1, "adjacent_find": 2, "is_sorted_until": 3,
               "all_of": 4, "any_of": 5, "none_of": 6, "is_sorted": 7}


def seg_query(x, offsets, query: str, op: str) -> np.ndarray:
    """verification/oracle/src/seg.rs:171-283: one u32 per segment (a count,
    a local index or the segment's length, or a 0 / 1 flag)."""
    x, off = _c(x), _c(offsets).astype(np.uint32)
    nseg = off.size - 1
    out = np.zeros(max(nseg, 0), np.uint32)
    opid = PRED2[op] if op in PRED2 else UNARY[op]
    if nseg > 0 and lib().orc_seg_query(_dt(x), _p(x), _p(off), nseg, SEG_QUERIES[query], opid,
                                        _p(out)) != 0:
        raise TypeError(x.dtype)
    return out


SEG_TRANSFORMS = {"filter": 0, "take": 1, "unique": 2, "reverse": 3, "adjacent_difference": 4}


def seg_transform(x, offsets, kind: str, param=0):
    """verification/oracle/src/seg.rs:41-153: (values, new offsets).  param:
    the predicate name (filter), k (take), the operator name
    (adjacent_difference)."""
    x, off = _c(x), _c(offsets).astype(np.uint32)
    nseg = off.size - 1
    out = np.empty_like(x)
    new_off = np.zeros(nseg + 1, np.uint32)
    if kind == "filter":
        p = UNARY[param]
    elif kind == "adjacent_difference":
        p = OPS[param]
    else:
        p = int(param)
    w = lib().orc_seg_transform(_dt(x), _p(x), _p(off), nseg, SEG_TRANSFORMS[kind], p, _p(out),
                                _p(new_off))
    if w < 0:
        raise TypeError(x.dtype)
    return out[:w], new_off
