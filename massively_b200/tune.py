"""Autotuner for kernel tile configurations, persisted per device and size.

The library compiles a few tile shapes per algorithm family (MB_TUNE_* in
include/massively_b200.h, listed by `mb_tune_config_count` /
`mb_tune_describe`).  `autotune()` times every shape on the caller's
workload with CUDA events and records the fastest in a JSON database keyed by
(device name, family, element type, log2 size bucket); `apply()` selects the
recorded shape on an executor.  Environment variables MB_TUNE_SCAN,
MB_TUNE_RADIX, MB_TUNE_REDUCE and MB_TUNE_SELECT force a configuration.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os

from . import _native as N
from .runtime import check

FAMILIES = {"scan": 0, "radix": 1, "reduce": 2, "select": 3}
DB_PATH = os.environ.get("MB_TUNE_DB",
                         os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_db.json"))


def configs(family: str) -> list[str]:
    L = N.lib()
    fid = FAMILIES[family]
    return [L.mb_tune_describe(fid, c).decode() for c in range(L.mb_tune_config_count(fid))]


def set_config(exec, family: str, config: int) -> None:
    check(N.lib().mb_tune_set(exec.handle, FAMILIES[family], int(config)))


def _key(device_name: str, family: str, dtype: str, n: int) -> str:
    bucket = int(math.log2(max(1, n)))
    return f"{device_name}|{family}|{dtype}|2^{bucket}"


def load_db(path: str = DB_PATH) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_db(db: dict, path: str = DB_PATH) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(exec, family: str, dtype: str, n: int, run, reps: int = 5, warmup: int = 2,
             path: str = DB_PATH) -> int:
    """Times `run()` (which enqueues one call of the family on `exec`) under
    every configuration; stores and selects the fastest."""
    import torch
    best, best_ms = -1, float("inf")
    timings = {}
    for c in range(N.lib().mb_tune_config_count(FAMILIES[family])):
        set_config(exec, family, c)
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        timings[c] = ms
        if ms < best_ms:
            best, best_ms = c, ms
    exec.sync()
    name = torch.cuda.get_device_name(exec.device)
    db = load_db(path)
    db[_key(name, family, dtype, n)] = {"config": best, "ms": best_ms,
                                        "timings_ms": timings,
                                        "describe": configs(family)[best]}
    save_db(db, path)
    set_config(exec, family, best)
    return best


def lookup(device_name: str, family: str, dtype: str, n: int, path: str = DB_PATH):
    rec = load_db(path).get(_key(device_name, family, dtype, n))
    return None if rec is None else int(rec["config"])


def apply(exec, dtype: str | None = None, n: int | None = None, path: str = DB_PATH) -> None:
    """Selects environment overrides, else recorded choices for (dtype, n)."""
    for fam, fid in FAMILIES.items():
        v = os.environ.get(f"MB_TUNE_{fam.upper()}")
        if v is not None:
            set_config(exec, fam, int(v))
            continue
        if dtype is not None and n is not None:
            import torch
            c = lookup(torch.cuda.get_device_name(exec.device), fam, dtype, n, path)
            if c is not None:
                set_config(exec, fam, c)
