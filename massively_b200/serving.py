"""Continuous-batching request loop over the primitive kernels.

Requests (sort_by_key u32/u32, inclusive_scan u32, reduce_by_key u32/f32)
arrive on a Poisson clock with sizes log-uniform on [2^10, 2^26] and wait in
a queue.  Whenever one of the loop's stream slots frees up, the head of the
queue is launched: alone if it is large, else together with every waiting
small request of its kind as one segmented launch (segment ids as the
leading sort key; `seg` inclusive scans; reduce_by_key whose runs also break
at request boundaries), so requests that arrive while the GPU is busy
accumulate into larger batches.  Launches are admitted while the device
bytes of everything in flight fit a memory budget, run on several CUDA
streams so their work overlaps, and retire when their completion events
fire.  Latency is completion time (CUDA events on a common reference) minus
arrival time.  `plain_dispatch` serves the same trace one request per launch
in arrival order, for comparison.

Results are the same alone and in the mix (tests/test_serving_gpu.py).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import lazy
from . import op as O
from .runtime import Executor, check

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
        # reduce_by_key and, when coalesced, each run's first row)
        return {SORT: 26, SCAN: 9, RBK: 32}[self.kind] * self.n


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


INPUTS = {SORT: (("keys", np.uint32), ("values", np.uint32)),
          SCAN: (("x", np.uint32),),
          RBK: (("keys", np.uint32), ("values", np.float32))}


def materialize_inputs(exec: Executor, r: Request, into: dict | None = None) -> None:
    """Device inputs of a request, from the PCG streams (no host copy),
    written into `into` (columns of r.n items, e.g. slices of a batch's
    buffers) or into fresh buffers."""
    from .vector import copy
    cols = into or {name: exec.alloc(dt, r.n) for name, dt in INPUTS[r.kind]}
    if r.kind == SORT:
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 0xFFFFFFFF, r.seed, 0,
                                            cols["keys"].to_col()))
        copy(exec, lazy.counting(0).take(r.n), cols["values"])
    elif r.kind == SCAN:
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 1000, r.seed, 0, cols["x"].to_col()))
    else:
        # keys 0 / 1 from the PCG stream: runs of adjacent equal keys with
        # irregular (geometric) lengths; values are integers below 2^16 held
        # as f32, so any run shorter than 256 sums exactly in f32
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, 1, r.seed ^ 0x5bd1e995, 0,
                                            cols["keys"].to_col()))
        v = exec.alloc(np.uint32, r.n)
        check(N.lib().mb_random_uniform_u32(exec.handle, 0, (1 << 16) - 1, r.seed, 0,
                                            v.to_col()))
        copy(exec, lazy.cast(v, np.float32), cols["values"])
    r.inputs = cols


def materialize_batch(exec: Executor, reqs: list[Request]) -> dict:
    """Inputs of a coalesced group, each request's written straight into its
    slice of the batch's columns."""
    total = sum(r.n for r in reqs)
    batch = {name: exec.alloc(dt, total) for name, dt in INPUTS[reqs[0].kind]}
    off = 0
    for r in reqs:
        materialize_inputs(exec, r, {k: v.slice(off, off + r.n) for k, v in batch.items()})
        off += r.n
    return batch


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


def _offsets(exec, reqs):
    off = np.zeros(len(reqs) + 1, np.uint32)
    off[1:] = np.cumsum([r.n for r in reqs])
    return exec.to_device(off), off


def run_coalesced(exec: Executor, reqs: list[Request], batch: dict):
    """Several small requests of one kind, whose inputs sit back to back in
    `batch` (materialize_batch), in one segmented launch.

    Returns None when every request's outputs are set, or a callable that
    sets them and may only be called once the launch's work has completed
    (reduce_by_key: where each request's runs start in the batch's output is
    known only on the device; it is copied to pinned host memory behind the
    launch and read when the launch retires)."""
    from . import seg, vector
    kind = reqs[0].kind
    dev_off, host_off = _offsets(exec, reqs)
    sgm = seg.Segmentation(dev_off, int(host_off[-1]))
    if kind == SCAN:
        x = batch["x"]
        y = seg.ForEachSegment(seg.InclusiveScan(O.Add)).run(exec, sgm.segments(x)).values()
        for i, r in enumerate(reqs):
            r.outputs = {"y": y.slice(int(host_off[i]), int(host_off[i + 1]))}
    elif kind == SORT:
        keys, vals = batch["keys"], batch["values"]
        ids = sgm.segment_ids(exec)
        from .iter import Zip
        out = vector.radix_sort_by_key(exec, Zip(ids, keys), Zip(keys, vals))
        sk, sv = out.into_columns()
        for i, r in enumerate(reqs):
            a, b = int(host_off[i]), int(host_off[i + 1])
            r.outputs = {"keys": sk.slice(a, b), "values": sv.slice(a, b)}
    else:
        keys, vals = batch["keys"], batch["values"]
        # Runs break at request boundaries as well as at key changes, and
        # come out grouped by request, in order.  A second value column
        # (MIN over the row index) gives each run's first row; request i's
        # runs then start at lower_bound(first rows, offset_i).
        k, v, first = _rbk_with_first_rows(exec, keys, vals, dev_off, int(host_off[-1]))
        starts = vector.lower_bound(exec, first, dev_off)
        host = torch.empty(len(reqs) + 1, dtype=torch.int32, pin_memory=True)
        host.copy_(starts.tensor.view(torch.int32), non_blocking=True)

        def finish():
            st = host.numpy()
            for i, r in enumerate(reqs):
                a, b = int(st[i]), int(st[i + 1])
                r.outputs = {"keys": k.slice(a, b), "values": v.slice(a, b)}
        return finish
    return None


def _rbk_with_first_rows(exec, keys, vals, dev_off, total):
    """reduce_by_key_segmented of `vals` (ADD) that also returns each run's
    first row index."""
    from . import vector
    from .iter import Zip
    k, z = vector.reduce_by_key_segmented(
        exec, keys, Zip(vals, lazy.counting(0).take(total)), O.Equal,
        (np.float32(0), np.uint32(0xFFFFFFFF)), (O.Add, O.Min), dev_off)
    v, first = z.into_columns()
    return k, v, first


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
          small_n: int = 1 << 20, max_batch: int = 256, streams: int = 8, depth: int = 4,
          keep_outputs: bool = False) -> ServeStats:
    """Continuous batching.  Arrived requests wait in a queue; whenever one
    of the `streams` launch slots (each holds up to `depth` launches in
    flight) frees up, the head of the queue is launched: alone if it is
    large, else together with every waiting small request of its kind (up to
    `max_batch`) as one segmented launch.  Requests that arrive while the
    GPU is busy therefore accumulate into larger batches.  A launch is
    admitted only while the bytes of everything in flight stay within
    `budget_bytes`; requests retire when their completion event fires."""
    exec.reserve_pool(budget_bytes)
    pool = [torch.cuda.Stream() for _ in range(streams)]
    clock = _Clock()
    # The queue in arrival order, plus one queue of small requests per kind
    # (a request leaves both when launched; the other copy is skipped
    # later), so forming a launch costs O(batch), not O(queue).
    queue: deque[Request] = deque()
    small: dict[str, deque[Request]] = {SORT: deque(), SCAN: deque(), RBK: deque()}
    taken: set[int] = set()
    nwait = 0
    inflight = []               # (event, [requests], bytes, stream index, finish)
    load = [0] * streams        # launches in flight per stream
    used = max_used = launches = nxt = done_count = 0

    def pop_live(q):
        while q and q[0].rid in taken:
            q.popleft()
        return q[0] if q else None

    while done_count < len(reqs):
        still = []
        for ev, group, b, si, finish in inflight:
            if ev.query():
                t = clock.gpu_time(ev)
                if finish is not None and keep_outputs:
                    finish()
                for r in group:
                    r.done = t
                    if not keep_outputs:
                        r.outputs = {}
                    r.inputs = {}
                used -= b
                done_count += len(group)
                load[si] -= 1
            else:
                still.append((ev, group, b, si, finish))
        inflight = still
        now = clock.now()
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            r = reqs[nxt]
            queue.append(r)
            if r.n <= small_n:
                small[r.kind].append(r)
            nwait += 1
            nxt += 1
        launched = False
        while nwait:
            si = min(range(streams), key=lambda i: load[i])
            if load[si] >= depth:
                break
            head = pop_live(queue)
            if head.n > small_n:
                group = [head]
            else:
                group, room, q = [], budget_bytes - used, small[head.kind]
                while len(group) < max_batch:
                    r = pop_live(q)
                    if r is None or (r.bytes_needed() > room and group):
                        break
                    q.popleft()
                    group.append(r)
                    room -= r.bytes_needed()
            b = sum(r.bytes_needed() for r in group)
            if used + b > budget_bytes and inflight:
                if len(group) > 1 or head.n <= small_n:
                    for r in reversed(group):  # back to the front of its queue
                        small[head.kind].appendleft(r)
                break               # wait for memory to come back
            for r in group:
                taken.add(r.rid)
            nwait -= len(group)
            with torch.cuda.stream(pool[si]):
                exec.bind_current_stream()
                finish = None
                if len(group) == 1:
                    materialize_inputs(exec, group[0])
                    run_single(exec, group[0])
                else:
                    finish = run_coalesced(exec, group, materialize_batch(exec, group))
                ev = torch.cuda.Event(enable_timing=True)
                ev.record()
            used += b
            max_used = max(max_used, used)
            load[si] += 1
            launches += 1
            launched = True
            inflight.append((ev, group, b, si, finish))
        if not launched:
            if not inflight and not nwait and nxt < len(reqs):
                time.sleep(max(0.0, min(1e-3, reqs[nxt].arrival - clock.now())))
            elif inflight:
                time.sleep(20e-6)
    exec.bind_current_stream()
    torch.cuda.synchronize()
    t_end = max(r.done for r in reqs)
    return _stats(reqs, t_end, launches, max_used)


def plain_dispatch(exec: Executor, reqs: list[Request], keep_outputs: bool = False,
                   wait: bool = True) -> ServeStats:
    """One request per launch, in arrival order, on one stream.  With `wait`
    (plain request/response serving) each request's result is waited for
    before the next request is dispatched; without it the requests are
    queued back to back on the stream, with no coalescing or overlap."""
    exec.reserve_pool(40 << 30)
    clock = _Clock()
    events = []
    for r in reqs:
        delay = r.arrival - clock.now()
        if delay > 0:
            time.sleep(delay)
        materialize_inputs(exec, r)
        run_single(exec, r)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        events.append(ev)
        if wait:
            ev.synchronize()
        if not keep_outputs:
            # stream-ordered frees: the memory is reused only by later work
            # on this stream
            r.inputs, r.outputs = {}, {}
    torch.cuda.synchronize()
    for r, ev in zip(reqs, events):
        r.done = clock.gpu_time(ev)
    t_end = max(r.done for r in reqs)
    return _stats(reqs, t_end, len(reqs), 0)
