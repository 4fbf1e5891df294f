"""Autotuner for kernel configurations, persisted per device and workload.

The library compiles a few configurations per algorithm family (MB_TUNE_* in
include/massively_b200.h, listed by `mb_tune_config_count` /
`mb_tune_describe`):

- radix: onesweep tile shape (threads per CTA, keys per thread), CTAs per
  SM, peer discovery (shared-memory lane masks or ballots) and 64-bit pair
  staging; the digit width is 8 bits in every configuration;
- scan: tile size and which warp runs the look-back;
- seg: ForEachSegment(Reduce) as tile-local folds or a carried look-back;
- reduce, select: one configuration each.

`autotune()` times every configuration of a family on the caller's workload
with CUDA events and records the fastest in a JSON database keyed by
(device name, family, element type, log2 size bucket, and -- for segmented
work -- a segment-length class: log2 of the mean length and the coefficient
of variation rounded to a half).  `apply()` selects the recorded choices for
a workload on an executor and returns them.  The database lives outside the
package (MB_TUNE_DB, else $XDG_CACHE_HOME/massively_b200/tune_db.json, else
~/.cache/massively_b200/tune_db.json).  Keys missing there fall back to a
read-only table shipped with the package (tune_table.json: choices measured
on a B200 for the benchmark's workloads, under the device name "*").  Environment variables MB_TUNE_SCAN,
MB_TUNE_RADIX, MB_TUNE_REDUCE, MB_TUNE_SELECT and MB_TUNE_SEG force a
configuration.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import _native as N
from .runtime import check

FAMILIES = {"scan": 0, "radix": 1, "reduce": 2, "select": 3, "seg": 4, "search": 5}


def default_db_path() -> str:
    p = os.environ.get("MB_TUNE_DB")
    if p:
        return p
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "massively_b200", "tune_db.json")


def configs(family: str) -> list[str]:
    L = N.lib()
    fid = FAMILIES[family]
    return [L.mb_tune_describe(fid, c).decode() for c in range(L.mb_tune_config_count(fid))]


def set_config(exec, family: str, config: int) -> None:
    check(N.lib().mb_tune_set(exec.handle, FAMILIES[family], int(config)))


def get_config(exec, family: str) -> int:
    return int(N.lib().mb_tune_get(exec.handle, FAMILIES[family]))


def segment_class(lengths) -> str:
    """Class of a segment-length distribution: log2 of the mean length and
    the coefficient of variation, rounded to a half ("" for no segments)."""
    x = np.asarray(lengths, dtype=np.float64)
    if x.size == 0:
        return ""
    mean = float(x.mean())
    cv = float(x.std() / mean) if mean > 0 else 0.0
    return f"seg:mean2^{int(round(math.log2(max(mean, 1.0))))}:cv{round(cv * 2) / 2:g}"


def _key(device_name: str, family: str, dtype: str, n: int, dist: str = "") -> str:
    bucket = int(math.log2(max(1, n)))
    k = f"{device_name}|{family}|{dtype}|2^{bucket}"
    return f"{k}|{dist}" if dist else k


def load_db(path: str | None = None) -> dict:
    try:
        with open(path or default_db_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_db(db: dict, path: str | None = None) -> None:
    path = path or default_db_path()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(exec, family: str, dtype: str, n: int, run, reps: int = 5, warmup: int = 2,
             path: str | None = None, dist: str = "") -> int:
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
    db[_key(name, family, dtype, n, dist)] = {"config": best, "ms": best_ms,
                                              "timings_ms": timings,
                                              "describe": configs(family)[best]}
    save_db(db, path)
    set_config(exec, family, best)
    return best


SHIPPED_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_table.json")


def lookup(device_name: str, family: str, dtype: str, n: int, path: str | None = None,
           dist: str = "", shipped: bool = False):
    rec = load_db(path).get(_key(device_name, family, dtype, n, dist))
    if rec is None and shipped:
        rec = load_db(SHIPPED_TABLE).get(_key("*", family, dtype, n, dist))
    return None if rec is None else int(rec["config"])


def apply(exec, dtype: str | None = None, n: int | None = None, path: str | None = None,
          dist: str = "") -> dict:
    """Selects, per family, an environment override, else the recorded
    choice for (dtype, n, dist) -- the caller's database, then the shipped
    table -- else the built-in default; returns {family: (config, source)}
    with source "env", "db", "shipped" or "default"."""
    chosen = {}
    name = None
    for fam, fid in FAMILIES.items():
        v = os.environ.get(f"MB_TUNE_{fam.upper()}")
        if v is not None:
            set_config(exec, fam, int(v))
            chosen[fam] = (int(v), "env")
            continue
        c = None
        if dtype is not None and n is not None:
            if name is None:
                import torch
                name = torch.cuda.get_device_name(exec.device)
            c = lookup(name, fam, dtype, n, path, dist)
            if c is None:
                c = lookup(name, fam, dtype, n, path, dist, shipped=True)
                src = "shipped"
            else:
                src = "db"
        if c is not None:
            set_config(exec, fam, c)
            chosen[fam] = (c, src)
        else:
            set_config(exec, fam, -1)
            chosen[fam] = (-1, "default")
    return chosen
