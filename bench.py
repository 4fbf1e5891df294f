"""Benchmark of the massively primitive path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--no-e2e] [--no-cpu] [--no-secondary]

Default workload: the large-vector configuration of massively's north-star
benchmark -- stable radix sort_by_key of 2^28 (u32 key, u32 value) pairs,
keys uniform 32-bit from massively's PCG stream (seed 0), values = index.
`value` is whole-job Gkeys/s with inputs resident in HBM; `e2e` is the same
metric through the public API with pinned host buffers and the host<->device
copies inside the timed region.  The other large-vector entries (u32 scan of
2^30, f32 scan of 2^28, copy_where of 2^28, 16-bit-key sort, u64 sort of
2^27) are measured in the same run and reported under `secondary`.

Multi-GPU (torchrun): every rank runs an independent replica on its own GPU
(the path has no exchange step); timing is the max over ranks and `value`
counts all ranks' keys.  `--impl reference` times the CPU oracle (the
sequential restatement of massively's own CPU reference) on rank 0 on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# torch and the kernels' scratch share the device's stream-ordered pool
# (set before torch first touches CUDA; see massively_b200/__init__.py).
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "backend:cudaMallocAsync")

FALLBACK_HBM_GBS = 6650.0


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# DRAM traffic per launch of each workload's dominant kernel from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum), scaled to a full
# launch; see profiles/ for the capture commands and figures.  None until
# captured.
NCU_TRAFFIC_BYTES = {
    # radix_onesweep_tma_kernel, one digit pass over 2^28 (u32, u32) pairs:
    # dram__bytes_read.sum 2,159,642,368 + dram__bytes_write.sum 2,129,241,600
    # (algorithmic 16 B/pair = 4,294,967,296)
    "sort_by_key_u32_u32_2^28": 4288883968,
}


# ---------------------------------------------------------------- inputs --
# Inputs come from the library's own PCG streams (massively's util::random
# integer streams) on the device; normals are made on the host once, by an
# f64 Box-Muller over the same streams, and uploaded.

def device_uniform_u32(ex, lo, hi, seed, n):
    import massively_b200 as mb
    from massively_b200 import _native as N
    v = ex.alloc(np.uint32, n)
    mb.runtime.check(N.lib().mb_random_uniform_u32(ex.handle, lo, hi, seed, 0, v.to_col()))
    return v


def host_normal_f32(ex, seed, n, chunk=1 << 26):
    """N(0,1) as f32: u1 = the low 32 bits, u2 = the high 32 bits of the
    full-range uniform_u64 stream of `seed` (24-bit mantissas, half-step
    offset), z = sqrt(-2 ln u1) cos(2 pi u2) in f64, rounded once."""
    import massively_b200 as mb
    from massively_b200 import _native as N
    out = np.empty(n, np.float32)
    for a in range(0, n, chunk):
        m = min(chunk, n - a)
        v = ex.alloc(np.uint64, m)
        mb.runtime.check(N.lib().mb_random_uniform_u64(ex.handle, 0, 0xFFFFFFFFFFFFFFFF, seed, a,
                                                      v.to_col()))
        bits = ex.to_host(v)
        u1 = ((bits & 0xFFFFFFFF) >> 8).astype(np.float64)
        u2 = (bits >> 40).astype(np.float64)
        u1 = (u1 + 0.5) * (1.0 / 16777216.0)
        u2 = (u2 + 0.5) * (1.0 / 16777216.0)
        out[a:a + m] = (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).astype(np.float32)
    return out


# ------------------------------------------------------------- workloads --

class Workload:
    name = ""
    metric = ""
    unit = ""
    dtype = ""
    kernel = ""
    family = None  # MB_KF_* id of the dominant kernel (per-kernel roofline)

    def family_bytes(self) -> float:  # algorithmic bytes of that kernel per step
        raise NotImplementedError

    def units(self) -> float:  # keys (or bytes) per step
        raise NotImplementedError

    def alg_bytes(self) -> float:
        raise NotImplementedError

    def value_from_ms(self, ms: float, n_gpus: int) -> float:
        raise NotImplementedError


class SortPairsU32(Workload):
    """Stable radix sort_by_key of (u32 key, u32 value) pairs, 8-bit onesweep
    byte model n * (4 + 2 * P * (4 + 4)), P = 4 digit passes (68 B/pair)."""

    kernel = "radix_onesweep_tma_kernel"

    def __init__(self, n=1 << 28, key_hi=0xFFFFFFFF, seed=0, tag=""):
        self.n, self.key_hi, self.seed = n, key_hi, seed
        bits = 32 if key_hi == 0xFFFFFFFF else int(key_hi).bit_length()
        self.passes = (bits + 7) // 8  # digit passes that move data (the others are skipped)
        self.name = f"sort_by_key_u32_u32_2^{int(np.log2(n))}{tag}"
        self.metric = "sort_by_key Gkeys/s"
        self.unit = "Gkeys/s"
        self.dtype = "u32"
        self.bits = bits

    def setup(self, ex):
        from massively_b200 import lazy
        import massively_b200 as mb
        from massively_b200 import _native as N
        self.keys = ex.alloc(np.uint32, self.n)
        mb.runtime.check(N.lib().mb_random_uniform_u32(ex.handle, 0, self.key_hi, self.seed, 0,
                                                      self.keys.to_col()))
        self.vals = ex.alloc(np.uint32, self.n)
        from massively_b200 import vector
        vector.copy(ex, lazy.counting(0).take(self.n), self.vals)
        self.ko = ex.alloc(np.uint32, self.n)
        self.vo = ex.alloc(np.uint32, self.n)

    def step(self, ex):
        import ctypes as C
        from massively_b200 import _native as N
        from massively_b200.runtime import check
        ks, vs = self.keys.to_src(), self.vals.to_src()
        check(N.lib().mb_radix_sort_by_key(ex.handle, C.byref(ks), 1, C.byref(vs), 1,
                                           C.byref(self.vo.to_col()), C.byref(self.ko.to_col())))

    def units(self):
        return float(self.n)

    def alg_bytes(self):
        return self.n * (4 + 2 * self.passes * (4 + 4))

    family = 0  # MB_KF_RADIX_ONESWEEP

    def family_bytes(self):
        return self.n * self.passes * 2 * (4 + 4)

    def value_from_ms(self, ms, n_gpus):
        return self.n * n_gpus / (ms * 1e-3) / 1e9

    def e2e(self, ex, host_k, host_v, out_v):
        from massively_b200 import vector
        dk = ex.to_device_pinned(host_k)
        dv = ex.to_device_pinned(host_v)
        sk, sv = vector.radix_sort_pairs(ex, dk, dv)
        ex.copy_to_pinned(sv, out_v)

    @staticmethod
    def e2e_device(ex, dk, dv):
        from massively_b200 import vector
        return vector.radix_sort_pairs(ex, dk, dv)[1]

    def host_inputs(self, ex):
        k = ex.to_host(device_uniform_u32(ex, 0, self.key_hi, self.seed, self.n))
        v = np.arange(self.n, dtype=np.uint32)
        return k, v

    def cpu(self, sample):
        from oracle import oracle as orc
        k = orc.uniform_u32(0, self.key_hi, self.seed, sample)
        v = np.arange(sample, dtype=np.uint32)
        t = time.perf_counter()
        orc.radix_sort_by_key([k], v)
        return time.perf_counter() - t, sample

    cpu_sample = 1 << 22


class ScanU32(Workload):
    """inclusive_scan (wrapping add) of 2^30 u32; bytes n * (4 + 4)."""

    kernel = "scan_smem_kernel"

    def __init__(self, n=1 << 30, seed=3):
        self.n, self.seed = n, seed
        self.name = f"inclusive_scan_u32_2^{int(np.log2(n))}"
        self.metric = "inclusive_scan GB/s"
        self.unit = "GB/s"
        self.dtype = "u32"

    def setup(self, ex):
        import massively_b200 as mb
        from massively_b200 import _native as N
        self.x = ex.alloc(np.uint32, self.n)
        mb.runtime.check(N.lib().mb_random_uniform_u32(ex.handle, 0, 0xFFFFFFFF, self.seed, 0,
                                                      self.x.to_col()))
        self.y = ex.alloc(np.uint32, self.n)

    def step(self, ex):
        import ctypes as C
        from massively_b200 import _native as N
        from massively_b200.runtime import check
        s = self.x.to_src()
        check(N.lib().mb_inclusive_scan(ex.handle, C.byref(s), 0, self.y.to_col()))

    def units(self):
        return self.alg_bytes()

    def alg_bytes(self):
        return self.n * 8.0

    family = 2  # MB_KF_SCAN

    def family_bytes(self):
        return self.alg_bytes()

    def value_from_ms(self, ms, n_gpus):
        return self.alg_bytes() * n_gpus / (ms * 1e-3) / 1e9

    def host_inputs(self, ex):
        return (ex.to_host(device_uniform_u32(ex, 0, 0xFFFFFFFF, self.seed, self.n)),)

    def e2e(self, ex, host_x, out_y):
        from massively_b200 import op, vector
        dx = ex.to_device_pinned(host_x)
        y = vector.inclusive_scan(ex, dx, op.Add)
        ex.copy_to_pinned(y, out_y)

    @staticmethod
    def e2e_device(ex, dx):
        from massively_b200 import op, vector
        return vector.inclusive_scan(ex, dx, op.Add)

    def cpu(self, sample):
        from oracle import oracle as orc
        x = orc.uniform_u32(0, 0xFFFFFFFF, self.seed, sample)
        t = time.perf_counter()
        orc.inclusive_scan(x, "add")
        return time.perf_counter() - t, sample * 8.0

    cpu_sample = 1 << 26


class ScanF32(ScanU32):
    """inclusive_scan (add) of 2^28 f32 N(0,1) (host Box-Muller bytes)."""

    def __init__(self, n=1 << 28, seed=4):
        super().__init__(n, seed)
        self.name = f"inclusive_scan_f32_2^{int(np.log2(n))}"
        self.dtype = "f32"

    def setup(self, ex):
        self.x = ex.to_device(host_normal_f32(ex, self.seed, self.n))
        self.y = ex.alloc(np.float32, self.n)

    def host_inputs(self, ex):
        return (host_normal_f32(ex, self.seed, self.n),)

    def cpu(self, sample):
        from oracle import oracle as orc
        x = orc.normal_f32(self.seed, sample)
        t = time.perf_counter()
        orc.inclusive_scan(x, "add")
        return time.perf_counter() - t, sample * 8.0


class CopyWhereU32(Workload):
    """copy_where of 2^28 u32 with the fused predicate key & 1 == 0 (~50%
    kept); bytes n * 4 + kept * 4."""

    kernel = "select_smem_kernel"

    def __init__(self, n=1 << 28, seed=5):
        self.n, self.seed = n, seed
        self.name = f"copy_where_u32_2^{int(np.log2(n))}"
        self.metric = "copy_where GB/s"
        self.unit = "GB/s"
        self.dtype = "u32"

    def setup(self, ex):
        import massively_b200 as mb
        from massively_b200 import _native as N
        self.x = ex.alloc(np.uint32, self.n)
        mb.runtime.check(N.lib().mb_random_uniform_u32(ex.handle, 0, 0xFFFFFFFF, self.seed, 0,
                                                      self.x.to_col()))
        self.y = ex.alloc(np.uint32, self.n)
        import torch
        self.cnt = torch.zeros(1, dtype=torch.uint32, device=self.x.tensor.device)
        self.step(ex)  # the exact kept count, for the byte model
        self.kept = int(self.cnt.cpu().item())

    def step(self, ex):
        import ctypes as C
        from massively_b200 import _native as N
        from massively_b200.runtime import check
        s = self.x.to_src()
        st = self.x.to_src()
        st.map, st.vtype = 3, 2  # IS_EVEN -> u32 flag
        check(N.lib().mb_copy_where(ex.handle, C.byref(s), 1, C.byref(st),
                                    C.byref(self.y.to_col()),
                                    C.cast(C.c_void_p(self.cnt.data_ptr()),
                                           C.POINTER(C.c_uint32)), None))

    def units(self):
        return self.alg_bytes()

    def alg_bytes(self):
        return self.n * 4.0 + self.kept * 4.0

    family = 3  # MB_KF_SELECT

    def family_bytes(self):
        return self.alg_bytes()

    def value_from_ms(self, ms, n_gpus):
        return self.alg_bytes() * n_gpus / (ms * 1e-3) / 1e9


class SortU64(Workload):
    """Keys-only radix sort of 2^27 u64 (uniform 64-bit, seed 2); 8-bit
    onesweep byte model n * (8 + 2 * 8 * 8) = 136 B/key."""

    kernel = "radix_onesweep_tma_kernel"

    def __init__(self, n=1 << 27, seed=2):
        self.n, self.seed = n, seed
        self.name = f"sort_u64_2^{int(np.log2(n))}"
        self.metric = "sort Gkeys/s"
        self.unit = "Gkeys/s"
        self.dtype = "u64"

    def setup(self, ex):
        import massively_b200 as mb
        from massively_b200 import _native as N
        self.keys = ex.alloc(np.uint64, self.n)
        mb.runtime.check(N.lib().mb_random_uniform_u64(ex.handle, 0, 0xFFFFFFFFFFFFFFFF,
                                                      self.seed, 0, self.keys.to_col()))
        self.ko = ex.alloc(np.uint64, self.n)

    def step(self, ex):
        import ctypes as C
        from massively_b200 import _native as N
        from massively_b200.runtime import check
        ks = self.keys.to_src()
        check(N.lib().mb_sort(ex.handle, C.byref(ks), 0, self.ko.to_col()))

    def units(self):
        return float(self.n)

    def alg_bytes(self):
        return self.n * (8 + 2 * 8 * 8)

    family = 0  # MB_KF_RADIX_ONESWEEP

    def family_bytes(self):
        return self.n * 8 * 2 * 8

    def value_from_ms(self, ms, n_gpus):
        return self.n * n_gpus / (ms * 1e-3) / 1e9


def lognormal_offsets(ex, nseg, total, seed, mu=3.0, sigma=1.5):
    """Segment offsets with lognormal(mu, sigma) lengths (host f64 Box-Muller
    over the PCG stream), scaled to sum to `total` by largest remainder;
    empty segments allowed."""
    z = host_normal_f32(ex, seed, nseg).astype(np.float64)
    raw = np.exp(mu + sigma * z)
    scaled = raw / raw.sum() * total
    base = np.floor(scaled).astype(np.int64)
    rem = total - int(base.sum())
    order = np.argsort(-(scaled - base), kind="stable")
    base[order[:rem]] += 1
    return np.concatenate([[0], np.cumsum(base)]).astype(np.uint32)


def zipf_keys(ex, n, nkeys, seed, s=1.1):
    """u32 keys Zipf(s) over `nkeys` distinct keys: rank r in [0, nkeys)
    from an inverse-CDF table (f64 weights (r+1)^-s, cumulated and scaled to
    2^32) over the full-range uniform_u32 stream of `seed`, then spread over
    the 32-bit space as rank * 2654435761 mod 2^32 (a bijection)."""
    import torch
    ranks = np.arange(1, nkeys + 1, dtype=np.float64)
    cdf = np.cumsum(ranks ** -s)
    cdf_u32 = np.minimum(np.floor(cdf / cdf[-1] * 2.0 ** 32), 2.0 ** 32 - 1).astype(np.int64)
    u = device_uniform_u32(ex, 0, 0xFFFFFFFF, seed, n).tensor.view(torch.int32)
    u = u.to(torch.int64) & 0xFFFFFFFF
    table = torch.from_numpy(cdf_u32).to(u.device)
    rank = torch.searchsorted(table, u, right=True).clamp_(max=nkeys - 1)
    keys = ex.alloc(np.uint32, n)
    keys.tensor.view(torch.int32).copy_((rank.to(torch.int64) * 2654435761 & 0xFFFFFFFF)
                                        .to(torch.int32))
    return keys


def bernoulli_flags(ex, n, p, seed):
    """u32 flags: 1 where the full-range uniform_u32 stream of `seed` is
    below floor(p * 2^32), else 0."""
    import torch
    fl = device_uniform_u32(ex, 0, 0xFFFFFFFF, seed, n)
    flag = ex.alloc(np.uint32, n)
    flag.tensor.view(torch.int32).copy_(
        ((fl.tensor.view(torch.int32).to(torch.int64) & 0xFFFFFFFF)
         < int(p * 2 ** 32)).to(torch.int32))
    return flag


class SegScanF32(Workload):
    """ForEachSegment(InclusiveScan(add)) of 2^26 f32 N(0,1) in 2^20 segments
    with lognormal(3, 1.5) lengths; bytes n * (4 + 4) + (S + 1) * 4."""

    kernel = "seg_kernel"

    def __init__(self, n=1 << 26, nseg=1 << 20, seed=6, mode="scan"):
        self.n, self.nseg, self.seed, self.mode = n, nseg, seed, mode
        lg = int(np.log2(n))
        self.name = {"scan": f"seg_inclusive_scan_f32_2^{lg}", "reduce": f"seg_reduce_f32_2^{lg}",
                     "sort": f"seg_sort_u32_2^{lg}",
                     "count_if": f"seg_count_if_f32_2^{lg}"}[mode] + \
            f"_in_2^{int(np.log2(nseg))}_segments"
        self.metric = "segmented GB/s"
        self.unit = "GB/s"
        self.dtype = "u32" if mode == "sort" else "f32"
        if mode == "sort":
            self.kernel = "ss_kernel"

    def setup(self, ex):
        from massively_b200 import seg
        off = lognormal_offsets(ex, self.nseg, self.n, self.seed + 100)
        self.sgm = seg.Segmentation.from_offsets(ex, ex.to_device(off))
        if self.mode == "sort":
            self.x = device_uniform_u32(ex, 0, 0xFFFFFFFF, self.seed, self.n)
        else:
            self.x = ex.to_device(host_normal_f32(ex, self.seed, self.n))

    def step(self, ex):
        from massively_b200 import op, seg
        it = self.sgm.segments(self.x)
        if self.mode == "scan":
            self.out = seg.ForEachSegment(seg.InclusiveScan(op.Add)).run(ex, it)
        elif self.mode == "reduce":
            self.out = seg.ForEachSegment(seg.Reduce(op.Add, np.float32(0))).run(ex, it)
        elif self.mode == "count_if":
            self.out = seg.ForEachSegment(seg.CountIf(op.IsPositive)).run(ex, it)
        else:
            self.out = seg.ForEachSegment(seg.Sort(op.Less)).run(ex, it)

    def units(self):
        return self.alg_bytes()

    def alg_bytes(self):
        offs = (self.nseg + 1) * 4.0
        if self.mode in ("reduce", "count_if"):
            return self.n * 4.0 + self.nseg * 4.0 + offs
        return self.n * 8.0 + offs  # scan; for the sort a one-pass lower bound

    def value_from_ms(self, ms, n_gpus):
        return self.alg_bytes() * n_gpus / (ms * 1e-3) / 1e9


class GroupByC4(Workload):
    """The group-by chain over 2^27 rows, replayed as one captured CUDA graph
    per step: copy_where of rows with flag (PCG < 0.3 * 2^32) -> radix sort of
    the kept (key, value) pairs -> reduce_by_key into (f32 sum, u32 count,
    f32 min) -> set_intersection of the distinct keys with a sorted 2^20 u32
    list.  Keys Zipf(1.1) over 2^20 keys (inverse-CDF table over the PCG
    uniform), values f32 N(0,1).  Bytes: the sum of the stages' byte models
    at the measured counts."""

    kernel = "group_by (graph)"

    def __init__(self, n=1 << 27, nkeys=1 << 20, seed=7):
        self.n, self.nkeys, self.seed = n, nkeys, seed
        self.name = f"group_by_2^{int(np.log2(n))}_rows"
        self.metric = "group-by GB/s"
        self.unit = "GB/s"
        self.dtype = "u32/f32"

    def setup(self, ex):
        import torch

        from massively_b200 import pipeline
        self.keys = zipf_keys(ex, self.n, self.nkeys, self.seed)
        torch.cuda.empty_cache()
        self.values = ex.to_device(host_normal_f32(ex, self.seed + 1, self.n))
        self.flag = bernoulli_flags(ex, self.n, 0.3, self.seed + 2)
        other = device_uniform_u32(ex, 0, 0xFFFFFFFF, self.seed + 3, 1 << 20)
        from massively_b200 import vector
        self.other = vector.sort(ex, other)
        self.cap = pipeline.Captured(
            ex, lambda e: pipeline.group_by(e, self.keys, self.values, self.flag, self.other))
        self.cap.replay()
        out = self.cap.outputs
        self.kept = out["kept"].logical_len()
        self.runs = out["keys"].logical_len()
        self.common = out["common"].logical_len()

    def step(self, ex):
        self.cap.replay()

    def units(self):
        return self.alg_bytes()

    def alg_bytes(self):
        n, m, r, L = self.n, self.kept, self.runs, 1 << 20
        select = n * 12.0 + m * 8.0           # key, value, flag in; kept rows out
        sort = m * (4 + 2 * 4 * 8.0)          # onesweep model, 4 passes
        rbk = m * 8.0 + r * 16.0              # sorted pairs in; key + 3 aggregates out
        inter = r * 4.0 + L * 4.0 + self.common * 4.0
        return select + sort + rbk + inter

    def value_from_ms(self, ms, n_gpus):
        return self.alg_bytes() * n_gpus / (ms * 1e-3) / 1e9


class SimpleWorkload(Workload):
    """A one-call step over resident inputs, reported in GB/s of its byte
    model: reduce (n * 4), merge of two sorted lists ((l + r) * 4 * 2),
    gather through a random permutation (n * 12: indices, the values they
    pick, the output), find_if with no passing item (a full scan, n * 4),
    minmax_element over f32 normals (n * 4) and scatter_reduce of u32 adds
    into 2^20 counters (n * 8 + 2^20 * 8); set_intersection / set_union of two
    sorted lists of n / 2 u32 uniform over [0, 2^27) ((l + r) * 4 in + the
    kept items * 4 out)."""

    kernel = "single call"

    def __init__(self, kind, n):
        self.kind, self.n = kind, n
        lg = int(np.log2(n))
        self.name = {"reduce": f"reduce_add_u32_2^{lg}", "merge": f"merge_u32_2x2^{lg - 1}",
                     "gather": f"gather_u32_2^{lg}",
                     "lower_bound": f"lower_bound_u32_2^{lg}_in_2^24",
                     "find_if": f"find_if_u32_2^{lg}_no_hit",
                     "scatter_reduce": f"scatter_reduce_add_u32_2^{lg}_into_2^20",
                     "minmax": f"minmax_element_f32_2^{lg}",
                     "set_intersection": f"set_intersection_u32_2x2^{lg - 1}",
                     "set_union": f"set_union_u32_2x2^{lg - 1}"}[kind]
        self.metric = f"{kind} GB/s"
        self.unit = "GB/s"
        self.dtype = "f32" if kind == "minmax" else "u32"

    def setup(self, ex):
        from massively_b200 import lazy, vector
        if self.kind == "reduce":
            self.x = device_uniform_u32(ex, 0, 0xFFFFFFFF, 8, self.n)
        elif self.kind == "merge":
            h = self.n // 2
            self.a = vector.sort(ex, device_uniform_u32(ex, 0, 0xFFFFFFFF, 9, h))
            self.b = vector.sort(ex, device_uniform_u32(ex, 0, 0xFFFFFFFF, 10, h))
        elif self.kind in ("set_intersection", "set_union"):
            h = self.n // 2
            self.a = vector.sort(ex, device_uniform_u32(ex, 0, (1 << 27) - 1, 19, h))
            self.b = vector.sort(ex, device_uniform_u32(ex, 0, (1 << 27) - 1, 20, h))
            fn = vector.set_intersection if self.kind == "set_intersection" else vector.set_union
            self.kept = fn(ex, self.a, self.b).logical_len()
        elif self.kind == "lower_bound":
            self.src = vector.sort(ex, device_uniform_u32(ex, 0, 0xFFFFFFFF, 13, 1 << 24))
            self.x = device_uniform_u32(ex, 0, 0xFFFFFFFF, 14, self.n)
        elif self.kind == "scatter_reduce":
            self.x = device_uniform_u32(ex, 0, 0xFFFF, 17, self.n)
            self.idx = device_uniform_u32(ex, 0, (1 << 20) - 1, 18, self.n)
            self.res = ex.alloc(np.uint32, 1 << 20)
        elif self.kind == "find_if":
            self.x = device_uniform_u32(ex, 1, 0xFFFFFFFF, 15, self.n)  # no zero: no hit
            self.res = ex.alloc(np.uint32, 2)
        elif self.kind == "minmax":
            self.x = ex.to_device(host_normal_f32(ex, 16, self.n))
            self.res = ex.alloc(np.uint32, 2)
        else:
            self.x = device_uniform_u32(ex, 0, 0xFFFFFFFF, 11, self.n)
            r = device_uniform_u32(ex, 0, 0xFFFFFFFF, 12, self.n)
            iota = ex.alloc(np.uint32, self.n)
            vector.copy(ex, lazy.counting(0).take(self.n), iota)
            self.idx = vector.radix_sort_by_key(ex, r, iota)  # a random permutation

    def step(self, ex):
        from massively_b200 import op, vector
        if self.kind == "reduce":
            self.out = vector.reduce_to_device(ex, self.x, np.uint32(0), op.Add)
        elif self.kind == "merge":
            self.out = vector.merge(ex, self.a, self.b)
        elif self.kind == "set_intersection":
            self.out = vector.set_intersection(ex, self.a, self.b)
        elif self.kind == "set_union":
            self.out = vector.set_union(ex, self.a, self.b)
        elif self.kind == "lower_bound":
            self.out = vector.lower_bound(ex, self.src, self.x)
        elif self.kind == "scatter_reduce":
            vector.scatter_reduce(ex, self.x, self.idx, np.uint32(0), op.Add, self.res)
        elif self.kind == "find_if":
            vector.find_if(ex, self.x, "is_false", out=self.res)
        elif self.kind == "minmax":
            vector.minmax_element(ex, self.x, out=self.res)
        else:
            self.out = vector.gather(ex, self.x, self.idx)

    def units(self):
        return self.alg_bytes()

    def alg_bytes(self):
        # lower_bound: each query's value in and index out (the 64 MB source
        # stays in L2 after the first probes)
        if self.kind == "scatter_reduce":  # value + index per proposal, 2^20 counters r+w
            return 8.0 * self.n + 8.0 * (1 << 20)
        if self.kind in ("set_intersection", "set_union"):
            return 4.0 * self.n + 4.0 * self.kept
        return {"reduce": 4.0, "merge": 8.0, "gather": 12.0, "lower_bound": 8.0, "find_if": 4.0,
                "minmax": 4.0}[self.kind] * self.n

    def value_from_ms(self, ms, n_gpus):
        return self.alg_bytes() * n_gpus / (ms * 1e-3) / 1e9


def _n(default_log2: int) -> int:
    """Items of a workload: its configured size, or 2^MB_BENCH_LOG2N for
    small profiling captures of the same kernels."""
    v = os.environ.get("MB_BENCH_LOG2N")
    return 1 << (int(v) if v else default_log2)


WORKLOADS = {
    "sort_pairs_u32": lambda: SortPairsU32(n=_n(28)),
    "sort_pairs_u32_16bit": lambda: SortPairsU32(n=_n(28), key_hi=65535, seed=1,
                                                 tag="_keys2^16"),
    "scan_u32": lambda: ScanU32(n=_n(30)),
    "scan_f32": lambda: ScanF32(n=_n(28)),
    "copy_where_u32": lambda: CopyWhereU32(n=_n(28)),
    "sort_u64": lambda: SortU64(n=_n(27)),
    "seg_scan_f32": lambda: SegScanF32(n=_n(26)),
    "seg_reduce_f32": lambda: SegScanF32(n=_n(26), mode="reduce"),
    "seg_sort_u32": lambda: SegScanF32(n=_n(26), mode="sort"),
    "seg_count_if_f32": lambda: SegScanF32(n=_n(26), mode="count_if"),
    "group_by": lambda: GroupByC4(n=_n(27)),
    "reduce_u32": lambda: SimpleWorkload("reduce", _n(30)),
    "merge_u32": lambda: SimpleWorkload("merge", _n(28)),
    "gather_u32": lambda: SimpleWorkload("gather", _n(28)),
    "lower_bound_u32": lambda: SimpleWorkload("lower_bound", _n(26)),
    "find_if_u32": lambda: SimpleWorkload("find_if", _n(28)),
    "scatter_reduce_u32": lambda: SimpleWorkload("scatter_reduce", _n(28)),
    "minmax_element_f32": lambda: SimpleWorkload("minmax", _n(28)),
    "set_intersection_u32": lambda: SimpleWorkload("set_intersection", _n(28)),
    "set_union_u32": lambda: SimpleWorkload("set_union", _n(28)),
}
SECONDARY = ["scan_u32", "scan_f32", "copy_where_u32", "sort_pairs_u32_16bit", "sort_u64",
             "seg_scan_f32", "seg_reduce_f32", "seg_sort_u32", "group_by", "reduce_u32",
             "merge_u32", "gather_u32", "lower_bound_u32", "find_if_u32",
             "minmax_element_f32", "scatter_reduce_u32", "seg_count_if_f32",
             "set_intersection_u32", "set_union_u32"]


# -------------------------------------------------------------- helpers --

class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.lines = device, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def time_steps(ex, wl, steps, warmup, dist, kernel_times=None):
    """CUDA-event time per step (max over ranks).  With `kernel_times` (a
    dict), the dominant kernel's launches inside the timed region are also
    bracketed by the library's own events (mb_kernel_timing) and their count
    and summed time stored there."""
    import ctypes as C

    import torch

    from massively_b200 import _native as N
    for _ in range(warmup):
        wl.step(ex)
    torch.cuda.synchronize()
    timing = kernel_times is not None and wl.family is not None
    if timing:
        for fam in range(4):  # forget anything recorded before
            N.lib().mb_kernel_timing_read(ex.handle, fam, None, None)
        N.lib().mb_kernel_timing(ex.handle, 1)
    if dist:
        import torch.distributed as D
        D.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        wl.step(ex)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    if timing:
        N.lib().mb_kernel_timing(ex.handle, 0)
        launches, kms = C.c_uint64(0), C.c_double(0.0)
        N.lib().mb_kernel_timing_read(ex.handle, wl.family, C.byref(launches), C.byref(kms))
        kernel_times["launches"] = int(launches.value)
        kernel_times["ms"] = float(kms.value)
    ex.sync()
    if dist:
        ms = max_over_ranks(ms, "cuda")
    return ms


def max_over_ranks(value: float, device: str) -> float:
    """The largest `value` of all ranks (every rank takes part; the
    whole job's time is its slowest rank's)."""
    import torch
    import torch.distributed as D
    t = torch.tensor([value], device=device, dtype=torch.float64)
    D.all_reduce(t, op=D.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(wl, budget_s=12.0):
    """The oracle on a bounded sample, repeated to ~budget_s of CPU work."""
    total_t, total_units, reps = 0.0, 0.0, 0
    sample = wl.cpu_sample
    while total_t < budget_s and reps < 50:
        t, u = wl.cpu(sample)
        total_t += t
        total_units += u
        reps += 1
    if wl.unit == "Gkeys/s":
        v = total_units / total_t / 1e9
    else:
        v = total_units / total_t / 1e9
    return {"value": v, "unit": wl.unit, "cores": 1, "kind": "port",
            "sample": f"{reps} x {sample} items of the same workload on 1 host core "
                      f"({os.cpu_count()} present); oracle/oracle.cpp, sequential, g++ -O3"}


def e2e_measure(ex, wl, steps):
    """Public API with pinned host buffers; every step uploads its inputs and
    downloads its result inside the timed region.  Workloads with a device
    function stream their steps through pipeline.run_host_batches (step i + 1
    uploads and step i - 1 downloads while step i computes); `sequential` is
    the same steps one at a time (upload, kernels, download, wait)."""
    import torch
    if not hasattr(wl, "e2e"):
        return None
    host = wl.host_inputs(ex)
    pinned = [torch.from_numpy(h.view(np.uint8)).pin_memory() for h in host]
    hv = [p.numpy().view(h.dtype) for p, h in zip(pinned, host)]
    outs_t = [torch.empty(host[-1].nbytes, dtype=torch.uint8).pin_memory() for _ in range(2)]
    outs = [o.numpy().view(host[-1].dtype) for o in outs_t]
    wl.e2e(ex, *hv, outs[0])  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        wl.e2e(ex, *hv, outs[0])
    torch.cuda.synchronize()
    dt_seq = (time.perf_counter() - t0) / steps
    h2d = sum(h.nbytes for h in host)
    d2h = host[-1].nbytes
    res = {"value": wl.value_from_ms(dt_seq * 1e3, 1), "unit": wl.unit,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}
    if hasattr(wl, "e2e_device"):
        from massively_b200 import pipeline
        batches = [tuple(hv)] * steps
        step_outs = [outs[i % 2] for i in range(steps)]
        pipeline.run_host_batches(ex, wl.e2e_device, batches[:2], step_outs[:2])  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pipeline.run_host_batches(ex, wl.e2e_device, batches, step_outs)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / steps
        res["value"] = wl.value_from_ms(dt * 1e3, 1)
        res["mode"] = (f"{steps} steps streamed through pipeline.run_host_batches (uploads, "
                       "kernels and downloads on three streams, two steps in flight)")
        res["sequential"] = {"value": wl.value_from_ms(dt_seq * 1e3, 1),
                             "mode": "one step at a time: upload, kernels, download, wait"}
    return res


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    torch.cuda.set_device(local)
    if dist:
        import datetime

        import torch.distributed as D
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                             device_id=torch.device(f"cuda:{local}"))
    import massively_b200 as mb
    ex = mb.Executor(local)
    from massively_b200 import tune
    wl = WORKLOADS[args.workload]()
    # the autotuner's recorded choice for this workload's (dtype, n), or an
    # MB_TUNE_<FAMILY> override, else the built-in default; reported below
    chosen = tune.apply(ex, wl.dtype, wl.n)
    tuning = {fam: {"config": c, "source": src,
                    "describe": tune.configs(fam)[c] if c >= 0 else "built-in default"}
              for fam, (c, src) in chosen.items()}
    wl.setup(ex)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    kt = {}
    ms = time_steps(ex, wl, args.steps, args.warmup, dist, kt)
    clocks = sampler.stop()
    value = wl.value_from_ms(ms, world)
    peak, peak_kind = measured_peak_hbm()
    step_achieved = wl.alg_bytes() / (ms * 1e-3) / 1e9
    # the dominant kernel alone: its algorithmic bytes over its own launches'
    # event-timed duration inside the timed region
    if wl.family is not None:
        achieved = wl.family_bytes() * args.steps / (kt["ms"] * 1e-3) / 1e9
    else:  # a multi-kernel step (segmented, group-by): its byte model over the step time
        achieved = step_achieved
        kt = {"launches": 0, "ms": 0.0}
    secondary = {}
    if not args.no_secondary and args.workload == "sort_pairs_u32":
        del wl.keys, wl.vals, wl.ko, wl.vo
        for name in SECONDARY:
            try:
                w2 = WORKLOADS[name]()
                # this workload's recorded tuning (the caller's database, then
                # the shipped table), else the built-in defaults
                ch2 = tune.apply(ex, w2.dtype, getattr(w2, "n", None))
                w2.setup(ex)
                kt2 = {}
                st2 = max(3, args.steps)
                ms2 = time_steps(ex, w2, st2, args.warmup, dist, kt2)
                if w2.family is not None:
                    a2 = w2.family_bytes() * st2 / (kt2["ms"] * 1e-3) / 1e9
                else:  # a multi-kernel step: its byte model over the step time
                    a2 = w2.alg_bytes() / (ms2 * 1e-3) / 1e9
                secondary[name] = {"metric": w2.metric, "value": w2.value_from_ms(ms2, world),
                                   "unit": w2.unit, "ms_per_step": ms2,
                                   "kernel": w2.kernel, "kernel_achieved_gbs": a2,
                                   "roofline_frac": a2 / peak,
                                   "step_achieved_gbs": w2.alg_bytes() / (ms2 * 1e-3) / 1e9}
                tuned = {f: {"config": c, "source": s} for f, (c, s) in ch2.items()
                         if s != "default"}
                if tuned:
                    secondary[name]["tuning"] = tuned
                del w2
                torch.cuda.empty_cache()
            except Exception as e:  # a secondary that is not built yet
                secondary[name] = {"error": str(e)[:200]}
        tune.apply(ex, wl.dtype, wl.n)  # back to the headline's choices
        # the serving loop on a shortened trace (MB_SERVE_SECONDS s of arrivals)
        try:
            torch.cuda.empty_cache()
            secs = float(os.environ.get("MB_SERVE_SECONDS", "1.0"))
            m = serving_measure(ex, secs, 1, rank, local)
            secondary["serving"] = {
                "metric": "batched-request requests/s (p50/p99 latency)",
                "value": m["ours"].req_per_s * world, "unit": "requests/s",
                "trace": {**{k: v for k, v in m["cfg"].items() if k != "mix"},
                          "mix": list(m["cfg"]["mix"]),
                          "note": f"{secs:g} s of arrivals (the configuration's 10 s trace "
                                  "shortened to keep the default run within minutes)"},
                "p50_ms": m["ours"].p50_ms, "p99_ms": m["ours"].p99_ms,
                "batched": _serve_stats(m["ours"]),
                "plain_dispatch": _serve_stats(m["plain"]),
                "queued_dispatch": _serve_stats(m["queued"]),
                "speedup_requests_per_s": m["ours"].req_per_s / m["plain"].req_per_s,
                "speedup_vs_queued": m["ours"].req_per_s / m["queued"].req_per_s,
                "clocks": m["clocks"]}
        except Exception as e:
            secondary["serving"] = {"error": str(e)[:200]}
    e2e = None
    if not args.no_e2e:
        try:
            torch.cuda.empty_cache()
            e2e = e2e_measure(ex, WORKLOADS[args.workload](), max(2, min(args.steps, 16)))
        except Exception as e:
            e2e = {"error": str(e)[:200]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(WORKLOADS[args.workload]())
    if rank == 0:
        line = {
            "metric": wl.metric, "value": value, "unit": wl.unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": wl.dtype, "data": "synthetic (massively PCG streams, seeded)",
            "config": {"workload": wl.name, "items_per_gpu": wl.n,
                       "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (no flush needed)",
                       "tuning": tuning},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": NCU_TRAFFIC_BYTES.get(wl.name),
                         "kernel": wl.kernel, "kernel_launches": kt["launches"],
                         "kernel_ms_per_launch": kt["ms"] / max(1, kt["launches"]),
                         "alg_bytes_per_launch": (wl.family_bytes() * args.steps
                                                  / max(1, kt["launches"]))
                                                 if wl.family is not None else None,
                         "step_achieved": step_achieved, "step_frac": step_achieved / peak,
                         "note": "achieved = the dominant kernel's algorithmic bytes / its "
                                 "CUDA-event time over the timed region; step_* = the whole "
                                 "step's algorithmic bytes / step time"},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": gpu_launches(wl, args.steps),
            "secondary": secondary or None,
        }
        print(json.dumps(line))
    if dist:
        import torch.distributed as D
        D.destroy_process_group()


def gpu_launches(wl, steps):
    """This library's kernels launched per step, times steps: a radix sort
    is one histogram + one plan kernel + one onesweep launch per key byte
    (4 for u32, 8 for u64; a pass whose digit is constant exits at once);
    scan and copy_where are one kernel each."""
    if isinstance(wl, SortPairsU32):
        per = 2 + 4
    elif isinstance(wl, SortU64):
        per = 2 + 8
    else:
        per = 1
    return per * steps


def _serve_stats(st):
    return {"requests_per_s": st.req_per_s, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
            "requests": st.requests, "launches": st.launches, "makespan_s": st.elapsed_s}


def serving_measure(ex, secs, warmup, seed, device):
    """The serving trace (Poisson 20k req/s for `secs` s of arrivals, mix
    60/25/15, n log-uniform on [2^10, 2^26], 40 GB budget) through the
    batched loop, awaited plain dispatch and queued plain dispatch, after a
    short warm-up of both loops (kernels loaded, the stream-ordered pool
    grown to its working size)."""
    import torch

    from massively_b200 import serving as S
    cfg = dict(rate=20_000.0, duration=secs, lo_log2=10, hi_log2=26, mix=(0.60, 0.25, 0.15))
    S.serve(ex, S.make_trace(**{**cfg, "duration": 0.1}, seed=99))
    for _ in range(max(1, warmup)):
        S.serve(ex, S.make_trace(**{**cfg, "duration": 0.01}, seed=98))
        S.plain_dispatch(ex, S.make_trace(**{**cfg, "duration": 0.01}, seed=98), wait=False)
    torch.cuda.synchronize()
    sampler = ClockSampler(device)
    sampler.start()
    ours = S.serve(ex, S.make_trace(**cfg, seed=seed))
    plain = S.plain_dispatch(ex, S.make_trace(**cfg, seed=seed), wait=True)
    queued = S.plain_dispatch(ex, S.make_trace(**cfg, seed=seed), wait=False)
    clocks = sampler.stop()
    ex.sync()
    return {"ours": ours, "plain": plain, "queued": queued, "clocks": clocks, "cfg": cfg}


def run_serving(args):
    """The batched request loop against plain one-request-per-launch
    dispatch on the same seeded trace: Poisson arrivals at 20k req/s, mix
    60% sort_by_key u32/u32, 25% inclusive_scan u32, 15% reduce_by_key
    u32/f32, n log-uniform on [2^10, 2^26], 40 GB admission budget.  The
    trace lasts MB_SERVE_SECONDS (default 1 s of arrivals, 20k requests);
    the arrival rate is above what one GPU completes, so both loops run
    saturated and requests/s is requests / makespan."""
    import torch

    import massively_b200 as mb
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ex = mb.Executor(local)
    secs = float(os.environ.get("MB_SERVE_SECONDS", "1.0"))
    m = serving_measure(ex, secs, args.warmup, rank, local)
    ours, plain, queued, clocks, cfg = m["ours"], m["plain"], m["queued"], m["clocks"], m["cfg"]
    if rank == 0:
        d = _serve_stats
        line = {
            "metric": "batched-request requests/s (p50/p99 latency)",
            "value": ours.req_per_s * world, "unit": "requests/s", "n_gpus": world,
            "steps": 1, "warmup": args.warmup, "ms_per_step": ours.elapsed_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32",
            "data": "synthetic (seeded Poisson trace, PCG inputs)",
            "config": {"workload": "serving", **{k: v for k, v in cfg.items() if k != "mix"},
                       "mix": list(cfg["mix"]), "budget_bytes": 40 << 30,
                       "parallelism": f"replicas{world}"},
            "p50_ms": ours.p50_ms, "p99_ms": ours.p99_ms,
            "batched": d(ours),
            "plain_dispatch": {**d(plain), "mode": "one request per launch, result awaited "
                                                  "before the next is dispatched"},
            "queued_dispatch": {**d(queued), "mode": "one request per launch, queued back to "
                                                    "back on one stream, no waiting"},
            "speedup_requests_per_s": ours.req_per_s / plain.req_per_s,
            "speedup_vs_queued": ours.req_per_s / queued.req_per_s,
            "clocks": clocks, "gpu_launches": ours.launches,
        }
        print(json.dumps(line))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "serving":
        print(json.dumps({"impl": "reference", "unavailable":
                          "massively has no request loop; plain_dispatch in the serving "
                          "line is the one-request-per-launch comparison"}))
        return
    wl = WORKLOADS[args.workload]()
    vals = []
    t_all, u_all = 0.0, 0.0
    for i in range(args.warmup + args.steps):
        t, u = wl.cpu(wl.cpu_sample)
        if i >= args.warmup:
            vals.append(t)
            t_all += t
            u_all += u
    v = u_all / t_all / 1e9
    line = {
        "impl": "reference", "metric": wl.metric, "value": v, "unit": wl.unit, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype,
        "data": "synthetic (massively PCG streams, seeded)",
        "config": {"workload": wl.name, "items_per_gpu": wl.n, "parallelism": "cpu",
                   "sample_items_per_step": wl.cpu_sample},
        "cpu_baseline": {"value": v, "unit": wl.unit, "cores": 1, "kind": "port",
                         "sample": f"{wl.cpu_sample} items per step; the C++ restatement of "
                                   "massively's sequential CPU oracle (its Rust oracle and "
                                   "CubeCL runtimes do not build offline)"},
        "e2e": {"value": v, "unit": wl.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=os.environ.get("MB_BENCH_WORKLOAD", "sort_pairs_u32"),
                    choices=sorted(WORKLOADS) + ["serving"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
