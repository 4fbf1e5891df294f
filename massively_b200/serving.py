"""Continuous-batching request loop over the primitive kernels.

Requests (sort_by_key u32/u32, inclusive_scan u32, reduce_by_key u32/f32)
arrive on a Poisson clock with sizes log-uniform on [2^10, 2^26].  The loop
admits arrived requests while their device buffers fit in a memory budget,
coalesces the small admitted requests of one kind into one segmented launch
(segment ids as the leading sort key, `seg` scans, or (segment, key)
run keys for reduce_by_key -- runs never cross request boundaries), runs
large requests on their own, keeps up to `streams` launches in flight on
separate CUDA streams, and retires requests when their completion event
fires.  Latency is completion time (from CUDA events on a common reference)
minus arrival time.  `plain_dispatch` serves the same trace one request per
launch in arrival order, for comparison.

Results are the same alone and in the mix: integer outputs bit-exact, f32
sums within the association bound (tests/test_serving_gpu.py).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import lazy
from . import op as O
from .runtime import DeviceVec, Executor, check

SORT, SCAN, RBK = "sort_by_key", "inclusive_scan", "reduce_by_key"


@dataclass
class Request:
    rid: int
    kind: str
    n: int
    arrival: float          # seconds after the trace start
    seed: int
    inputs: dict = field(default_factory=dict)
    outputs: dict = field(default_factory=dict)
    done: float = math.nan  # completion, seconds after the trace start

    def bytes_needed(self) -> int:
        # inputs + outputs + the kernels' scratch on the device (the sort's
        # ping-pong buffers and look-back states, the run-count scratch of
        # reduce_by_key)
        return {SORT: 26, SCAN: 9, RBK: 28}[self.kind] * self.n


def make_trace(rate: float = 20_000.0, duration: float = 1.0, lo_log2: int = 10,
               hi_log2: int = 26, mix=(0.60, 0.25, 0.15), seed: int = 0,
               max_requests: int | None = None) -> list[Request]:
    """Seeded Poisson arrivals with log-uniform sizes and the request mix."""
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    kinds = [SORT, SCAN, RBK]
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and len(reqs) >= max_requests):
            break
        n = int(2 ** rng.uniform(lo_log2, hi_log2))
        kind = kinds[int(rng.choice(3, p=np.asarray(mix) / np.sum(mix)))]
        reqs.append(Request(len(reqs), kind, n, t, int(rng.integers(1 << 31))))
    return reqs


def materialize_inputs(exec: Executor, r: Request) -> None:
    """Device inputs of a request, from the PCG streams (no host copy)."""
    from .vector import copy
    if r.kind == SORT:
        k = exec.alloc(np.uint32, r.n)
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 0xFFFFFFFF, r.seed, 0, k.to_col()))
        v = exec.alloc(np.uint32, r.n)
        copy(exec, lazy.counting(0).take(r.n), v)
        r.inputs = {"keys": k, "values": v}
    elif r.kind == SCAN:
        x = exec.alloc(np.uint32, r.n)
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 1000, r.seed, 0, x.to_col()))
        r.inputs = {"x": x}
    else:
        # sorted keys in runs of 8 (the group-by shape after sort_by_key)
        kk = exec.alloc(np.uint32, r.n)
        copy(exec, lazy.RepeatEach(lazy.counting(r.seed & 0xFFFF).take((r.n + 7) // 8), r.n,
                                   a=8), kk)
        v = exec.alloc(np.uint32, r.n)
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 1 << 20, r.seed, 0, v.to_col()))
        vf = exec.alloc(np.float32, r.n)
        copy(exec, lazy.cast(v, np.float32), vf)
        r.inputs = {"keys": kk, "values": vf}


# ------------------------------------------------------------ executors ----

def run_single(exec: Executor, r: Request) -> None:
    """One request, one set of launches (plain dispatch)."""
    from . import vector
    if r.kind == SORT:
        sk, sv = vector.radix_sort_pairs(exec, r.inputs["keys"], r.inputs["values"])
        r.outputs = {"keys": sk, "values": sv}
    elif r.kind == SCAN:
        r.outputs = {"y": vector.inclusive_scan(exec, r.inputs["x"], O.Add)}
    else:
        k, v = vector.reduce_by_key(exec, r.inputs["keys"], r.inputs["values"], O.Equal,
                                    np.float32(0), O.Add)
        r.outputs = {"keys": k, "values": v}


def _concat(exec, cols):
    total = sum(len(c) for c in cols)
    out = exec.alloc(cols[0].dtype, total)
    off = 0
    for c in cols:
        out.tensor[off:off + len(c)].copy_(c.tensor)
        off += len(c)
    return out


def _offsets(exec, reqs):
    off = np.zeros(len(reqs) + 1, np.uint32)
    off[1:] = np.cumsum([r.n for r in reqs])
    return exec.to_device(off), off


def run_coalesced(exec: Executor, reqs: list[Request]) -> None:
    """Several small requests of one kind in one segmented launch."""
    from . import seg, vector
    kind = reqs[0].kind
    dev_off, host_off = _offsets(exec, reqs)
    sgm = seg.Segmentation(dev_off, int(host_off[-1]))
    if kind == SCAN:
        x = _concat(exec, [r.inputs["x"] for r in reqs])
        y = seg.ForEachSegment(seg.InclusiveScan(O.Add)).run(exec, sgm.segments(x)).values()
        for i, r in enumerate(reqs):
            r.outputs = {"y": y.slice(int(host_off[i]), int(host_off[i + 1]))}
    elif kind == SORT:
        keys = _concat(exec, [r.inputs["keys"] for r in reqs])
        vals = _concat(exec, [r.inputs["values"] for r in reqs])
        ids = sgm.segment_ids(exec)
        from .iter import Zip
        out = vector.radix_sort_by_key(exec, Zip(ids, keys), Zip(keys, vals))
        sk, sv = out.into_columns()
        for i, r in enumerate(reqs):
            a, b = int(host_off[i]), int(host_off[i + 1])
            r.outputs = {"keys": sk.slice(a, b), "values": sv.slice(a, b)}
    else:
        keys = _concat(exec, [r.inputs["keys"] for r in reqs])
        vals = _concat(exec, [r.inputs["values"] for r in reqs])
        # runs break at request boundaries as well as at key changes
        k, v = vector.reduce_by_key_segmented(exec, keys, vals, O.Equal, np.float32(0), O.Add,
                                              dev_off)
        # runs come out grouped by request, in order; the synthetic keys hold
        # runs of 8, so request i owns ceil(n_i / 8) of them
        counts = [int(math.ceil(r.n / 8)) for r in reqs]
        starts = np.concatenate([[0], np.cumsum(counts)])
        for i, r in enumerate(reqs):
            a, b = int(starts[i]), int(starts[i + 1])
            r.outputs = {"keys": k.slice(a, b), "values": v.slice(a, b)}


# ---------------------------------------------------------------- loops ----

@dataclass
class ServeStats:
    requests: int
    elapsed_s: float
    req_per_s: float
    p50_ms: float
    p99_ms: float
    launches: int
    max_inflight_bytes: int


def _stats(reqs, t_end, launches, max_bytes) -> ServeStats:
    lat = np.array([(r.done - r.arrival) * 1e3 for r in reqs])
    return ServeStats(len(reqs), t_end, len(reqs) / t_end, float(np.percentile(lat, 50)),
                      float(np.percentile(lat, 99)), launches, max_bytes)


class _Clock:
    """Host clock for arrivals; GPU completion times on the same axis via a
    reference event recorded at the start."""

    def __init__(self):
        torch.cuda.synchronize()
        self.ref = torch.cuda.Event(enable_timing=True)
        self.ref.record()
        torch.cuda.synchronize()
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def gpu_time(self, ev) -> float:
        return self.ref.elapsed_time(ev) / 1e3


def serve(exec: Executor, reqs: list[Request], budget_bytes: int = 40 << 30,
          small_n: int = 1 << 20, max_batch: int = 256, streams: int = 4,
          keep_outputs: bool = False) -> ServeStats:
    """Continuous batching: admit by memory, coalesce small requests, keep
    `streams` launches in flight, retire on completion events."""
    pool = [torch.cuda.Stream() for _ in range(streams)]
    clock = _Clock()
    pending = list(reqs)        # in arrival order
    inflight = []               # (event, [requests], bytes, stream index)
    used = 0
    max_used = 0
    launches = 0
    nxt = 0
    done_count = 0
    busy = [False] * streams
    while done_count < len(reqs):
        # retire finished launches
        still = []
        for ev, group, b, si in inflight:
            if ev.query():
                t = clock.gpu_time(ev)
                for r in group:
                    r.done = t
                    if not keep_outputs:
                        r.outputs = {}
                    r.inputs = {}
                used -= b
                done_count += len(group)
                busy[si] = False
            else:
                still.append((ev, group, b, si))
        inflight = still
        # admit arrived requests while memory allows
        now = clock.now()
        admitted = []
        while nxt < len(pending) and pending[nxt].arrival <= now:
            r = pending[nxt]
            if used + r.bytes_needed() > budget_bytes and (inflight or admitted):
                break
            admitted.append(r)
            used += r.bytes_needed()
            nxt += 1
        max_used = max(max_used, used)
        if not admitted:
            if not inflight and nxt < len(pending):
                time.sleep(max(0.0, min(1e-3, pending[nxt].arrival - clock.now())))
            continue
        # group: small requests of a kind coalesce, large ones go alone
        groups = []
        for kind in (SORT, SCAN, RBK):
            small = [r for r in admitted if r.kind == kind and r.n <= small_n]
            for i in range(0, len(small), max_batch):
                groups.append(small[i:i + max_batch])
            groups += [[r] for r in admitted if r.kind == kind and r.n > small_n]
        for group in groups:
            si = next((i for i in range(streams) if not busy[i]), None)
            if si is None:  # all streams busy: queue behind the least-loaded one
                si = launches % streams
            busy[si] = True
            with torch.cuda.stream(pool[si]):
                exec.bind_current_stream()
                for r in group:
                    materialize_inputs(exec, r)
                if len(group) == 1:
                    run_single(exec, group[0])
                else:
                    run_coalesced(exec, group)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record()
            launches += 1
            inflight.append((ev, group, sum(r.bytes_needed() for r in group), si))
    exec.bind_current_stream()
    torch.cuda.synchronize()
    t_end = max(r.done for r in reqs)
    return _stats(reqs, t_end, launches, max_used)


def plain_dispatch(exec: Executor, reqs: list[Request], keep_outputs: bool = False) -> ServeStats:
    """One request per launch, in arrival order, on one stream."""
    clock = _Clock()
    events = []
    for r in reqs:
        wait = r.arrival - clock.now()
        if wait > 0:
            time.sleep(wait)
        materialize_inputs(exec, r)
        run_single(exec, r)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        events.append(ev)
        if not keep_outputs:
            # stream-ordered frees: the memory is reused only by later work
            # on this stream
            r.inputs, r.outputs = {}, {}
    torch.cuda.synchronize()
    for r, ev in zip(reqs, events):
        r.done = clock.gpu_time(ev)
    t_end = max(r.done for r in reqs)
    return _stats(reqs, t_end, len(reqs), 0)
