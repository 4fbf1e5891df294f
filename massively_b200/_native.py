"""ctypes binding of libmassively_b200.so (the C ABI of include/massively_b200.h).

The library is built in-tree by massively_b200/build.py.  There is no
fallback: if the shared library is missing or cannot be loaded, every entry
point raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmassively_b200.so")

# ----------------------------------------------------------------- ids -----

U8, U16, U32, U64, I8, I16, I32, I64, F32, F64 = range(10)
OK, LENGTH_MISMATCH, OUTPUT_TOO_SHORT, LENGTH_TOO_LARGE, INVALID_SEGMENTATION, \
    UNBOUND_COLUMN, FOREIGN_EXECUTOR, LAUNCH = range(8)
SRC_COLUMN, SRC_CONSTANT, SRC_COUNTING, SRC_STRIDE, SRC_PERMUTE, SRC_REVERSE, \
    SRC_REPEAT_EACH, SRC_TILE, SRC_ADJACENT = range(9)
KF_RADIX_ONESWEEP, KF_RADIX_HISTOGRAM, KF_SCAN, KF_SELECT, KF_SEARCH = range(5)


class mb_src(C.Structure):
    _fields_ = [("kind", C.c_int32), ("dtype", C.c_int32), ("vtype", C.c_int32),
                ("map", C.c_int32), ("data", C.c_void_p), ("index", C.c_void_p),
                ("len", C.c_uint64), ("a", C.c_uint64), ("b", C.c_uint64),
                ("owner", C.c_uint64), ("len_dev", C.c_void_p)]


class mb_col(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("pad_", C.c_int32),
                ("len", C.c_uint64), ("owner", C.c_uint64)]


class mb_error_detail(C.Structure):
    _fields_ = [("left", C.c_uint64), ("right", C.c_uint64)]


_lib = None
_P = C.POINTER


def _declare(L: C.CDLL) -> None:
    vp, u64, i32, u32 = C.c_void_p, C.c_uint64, C.c_int, C.c_uint32
    src, col = _P(mb_src), mb_col
    pcol = _P(mb_col)
    pu32 = _P(C.c_uint32)
    sig = {
        "mb_last_error_message": (C.c_char_p, []),
        "mb_last_error_detail": (None, [_P(mb_error_detail)]),
        "mb_abi_version": (i32, []),
        "mb_executor_create": (i32, [i32, _P(vp)]),
        "mb_executor_destroy": (i32, [vp]),
        "mb_executor_id": (u64, [vp]),
        "mb_sync": (i32, [vp]),
        "mb_get_stream": (i32, [vp, _P(vp)]),
        "mb_set_stream": (i32, [vp, vp]),
        "mb_use_own_stream": (i32, [vp]),
        "mb_alloc": (i32, [vp, u64, _P(vp)]),
        "mb_free": (i32, [vp, vp]),
        "mb_copy_to_device": (i32, [vp, vp, vp, u64]),
        "mb_copy_to_host": (i32, [vp, vp, vp, u64]),
        "mb_pool_stats": (i32, [vp, _P(u64), _P(u64)]),
        "mb_copy": (i32, [vp, src, col]),
        "mb_fill": (i32, [vp, vp, col]),
        "mb_replace_where": (i32, [vp, _P(u64), src, pcol, i32]),
        "mb_check_bounded_waits": (i32, [vp, i32]),
        "mb_transform_where": (i32, [vp, src, i32, src, pcol]),
        "mb_inclusive_scan": (i32, [vp, src, i32, col]),
        "mb_inclusive_scan_noalloc": (i32, [vp, src, i32, col]),
        "mb_exclusive_scan": (i32, [vp, src, i32, vp, col]),
        "mb_reduce": (i32, [vp, src, i32, vp, vp, vp]),
        "mb_copy_where": (i32, [vp, src, i32, src, pcol, pu32, pu32]),
        "mb_remove_where": (i32, [vp, src, i32, src, pcol, pu32, pu32]),
        "mb_partition": (i32, [vp, src, i32, i32, i32, pcol, pu32, pu32]),
        "mb_gather": (i32, [vp, src, src, src, col]),
        "mb_scatter": (i32, [vp, src, src, src, col]),
        "mb_radix_sort_by_key": (i32, [vp, src, i32, src, i32, pcol, pcol]),
        "mb_sort": (i32, [vp, src, i32, col]),
        "mb_sort_by_key": (i32, [vp, src, i32, src, i32, pcol, pcol]),
        "mb_reduce_by_key": (i32, [vp, src, i32, src, i32, _P(C.c_int), _P(u64), col, pcol,
                                   pu32, pu32]),
        "mb_reduce_by_key_segmented": (i32, [vp, src, i32, src, i32, _P(C.c_int), _P(u64), vp,
                                             u64, col, pcol, pu32, pu32]),
        "mb_inclusive_scan_by_key": (i32, [vp, src, i32, src, i32, col]),
        "mb_exclusive_scan_by_key": (i32, [vp, src, i32, src, i32, vp, col]),
        "mb_merge": (i32, [vp, src, src, i32, col]),
        "mb_lower_bound": (i32, [vp, src, src, i32, col]),
        "mb_unique": (i32, [vp, src, i32, col, pu32, pu32]),
        "mb_scatter_reduce": (i32, [vp, src, i32, src, _P(C.c_int), _P(C.c_uint64), _P(mb_col)]),
        "mb_seg_query": (i32, [vp, src, vp, u64, i32, i32, col]),
        "mb_seg_reverse": (i32, [vp, src, vp, u64, col]),
        "mb_seg_adjacent_difference": (i32, [vp, src, vp, u64, i32, col]),
        "mb_seg_keep": (i32, [vp, src, vp, u64, i32, i32, col, vp, pu32, pu32]),
        "mb_user_op_compile": (i32, [vp, i32, C.c_char_p, C.c_char_p, _P(vp)]),
        "mb_user_map_compile": (i32, [vp, i32, i32, C.c_char_p, C.c_char_p, _P(vp)]),
        "mb_user_op_check": (i32, [i32, i32, i32, C.c_char_p, C.c_char_p]),
        "mb_user_pred_compile": (i32, [vp, i32, C.c_char_p, C.c_char_p, _P(vp)]),
        "mb_sort_user": (i32, [vp, src, vp, src, i32, col, pcol]),
        "mb_user_op_destroy": (i32, [vp]),
        "mb_reduce_user": (i32, [vp, src, vp, vp, vp, vp]),
        "mb_inclusive_scan_user": (i32, [vp, src, vp, col]),
        "mb_exclusive_scan_user": (i32, [vp, src, vp, vp, col]),
        "mb_map_user": (i32, [vp, src, vp, col]),
        "mb_find_if": (i32, [vp, src, i32, pu32, pu32]),
        "mb_is_partitioned": (i32, [vp, src, i32, pu32, pu32]),
        "mb_adjacent_find": (i32, [vp, src, i32, pu32, pu32]),
        "mb_is_sorted_until": (i32, [vp, src, i32, pu32, pu32]),
        "mb_find_first_of": (i32, [vp, src, src, i32, pu32, pu32]),
        "mb_mismatch": (i32, [vp, src, src, i32, pu32, pu32]),
        "mb_equal": (i32, [vp, src, src, i32, pu32, pu32]),
        "mb_lexicographical_compare": (i32, [vp, src, src, i32, pu32, pu32]),
        "mb_min_element": (i32, [vp, src, i32, pu32, pu32]),
        "mb_max_element": (i32, [vp, src, i32, pu32, pu32]),
        "mb_minmax_element": (i32, [vp, src, i32, pu32, pu32]),
        "mb_unique_by_key": (i32, [vp, src, src, i32, i32, pcol, pu32, pu32]),
        "mb_upper_bound": (i32, [vp, src, src, i32, col]),
        "mb_merge_by_key": (i32, [vp, src, src, src, src, i32, i32, col, pcol]),
        "mb_set_union": (i32, [vp, src, src, i32, col, pu32, pu32]),
        "mb_set_intersection": (i32, [vp, src, src, i32, col, pu32, pu32]),
        "mb_set_difference": (i32, [vp, src, src, i32, col, pu32, pu32]),
        "mb_segmentation_validate_offsets": (i32, [vp, vp, u64, pu32]),
        "mb_segmentation_from_lengths": (i32, [vp, src, vp, pu32]),
        "mb_segmentation_segment_ids": (i32, [vp, vp, u64, vp, u64]),
        "mb_segmentation_lengths": (i32, [vp, vp, u64, vp]),
        "mb_segmentation_local_indices": (i32, [vp, vp, u64, vp, u64]),
        "mb_segmentation_from_segment_ids": (i32, [vp, src, u64, vp]),
        "mb_seg_inclusive_scan": (i32, [vp, src, vp, u64, i32, col]),
        "mb_seg_exclusive_scan": (i32, [vp, src, vp, u64, i32, vp, col]),
        "mb_seg_reduce": (i32, [vp, src, vp, u64, i32, vp, col]),
        "mb_seg_sort": (i32, [vp, src, vp, u64, i32, col]),
        "mb_random_uniform_u32": (i32, [vp, u32, u32, u64, u64, col]),
        "mb_random_uniform_u64": (i32, [vp, u64, u64, u64, u64, col]),
        "mb_graph_begin": (i32, [vp]),
        "mb_graph_end": (i32, [vp, _P(vp)]),
        "mb_graph_launch": (i32, [vp, vp]),
        "mb_graph_destroy": (i32, [vp]),
        "mb_tune_config_count": (i32, [i32]),
        "mb_tune_set": (i32, [vp, i32, i32]),
        "mb_tune_get": (i32, [vp, i32]),
        "mb_tune_describe": (C.c_char_p, [i32, i32]),
        "mb_kernel_timing": (i32, [vp, i32]),
        "mb_kernel_timing_read": (i32, [vp, i32, _P(u64), _P(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args


def exported_symbols() -> list[str]:
    """Every mb_* symbol declared in include/massively_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "massively_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", text)))


def lib() -> C.CDLL:
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m massively_b200.build` "
                "(there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def last_error() -> tuple[str, int, int]:
    L = lib()
    d = mb_error_detail()
    L.mb_last_error_detail(C.byref(d))
    return L.mb_last_error_message().decode(), int(d.left), int(d.right)
