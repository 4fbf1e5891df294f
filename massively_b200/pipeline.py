"""Multi-step pipelines over device counts, and their capture as CUDA graphs.

`group_by` is the filter -> sort -> aggregate -> join chain of the group-by
configuration: rows whose flag is set are kept (copy_where, count left on the
device), sorted by key (the sort reads that count on the device), reduced per
key run into (sum, count, min) (reduce_by_key with a constant-one column), and
the distinct keys are intersected with a sorted list (set_intersection).  No
step reads a count back to the host, so the whole chain can be captured once
and replayed: `Captured` records it into a CUDA graph (torch's graph capture,
with the executor bound to the capturing stream; the library's stream-ordered
scratch becomes graph allocations) and `replay` relaunches every kernel with
one call.  Inputs are read from the buffers given at capture time, so new
data is copied into those buffers before a replay.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lazy, vector
from . import op as O
from .iter import Zip
from .runtime import DeviceVec, Executor


def group_by(exec: Executor, keys: DeviceVec, values: DeviceVec, flag: DeviceVec,
             other: DeviceVec) -> dict:
    """keys u32, values f32, flag u32 (non-zero = keep), other sorted u32.
    Returns device vectors (each with its count on the device): the distinct
    kept keys in order, per key the f32 sum, u32 count and f32 min of its
    values, and the distinct keys also present in `other`."""
    kept = vector.copy_where(exec, Zip(keys, values), flag)
    k1, v1 = kept.cols
    sk, sv = vector.radix_sort_pairs(exec, k1, v1)
    ones = lazy.constant(1, np.uint32).take(len(sk))
    rk, agg = vector.reduce_by_key(exec, sk, Zip(sv, ones, sv), O.Equal,
                                   (np.float32(0), np.uint32(0), np.float32(np.inf)),
                                   (O.Add, O.Add, O.Min))
    s, c, m = agg.cols
    common = vector.set_intersection(exec, rk, other)
    return {"keys": rk, "sum": s, "count": c, "min": m, "common": common,
            "kept": k1}


class Captured:
    """`fn(exec)` captured once into a CUDA graph; `replay()` relaunches it on
    the current stream.  The outputs `fn` returned are kept (their buffers
    are rewritten by each replay).

    Every buffer the calls allocate (outputs, intermediates, device counts)
    is a slice of one arena (runtime.Arena) that this object owns: a warm-up
    run records the sizes, the arena is allocated before capture, and the
    captured calls take their storage from it.  So no allocation of torch's
    happens inside the capture, the outputs live exactly as long as the
    graph that writes them, and `release()` (or dropping this object) frees
    graph and buffers together.  The library's own per-call scratch is
    stream-ordered pool memory, which the capture turns into graph
    allocations."""

    def __init__(self, exec: Executor, fn, warmup: int = 1):
        from .runtime import Arena
        self.exec = exec
        self.arena = Arena()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            exec.bind_current_stream()
            with self.arena.on(exec):  # records the sizes of every allocation
                fn(exec)
            for _ in range(warmup - 1):  # loads kernels and fills the pools outside capture
                fn(exec)
        torch.cuda.current_stream().wait_stream(side)
        exec.sync()
        self.arena.allocate(exec.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            exec.bind_current_stream()
            with self.arena.on(exec):
                self.outputs = fn(exec)
        exec.bind_current_stream()

    def replay(self) -> None:
        self.graph.replay()

    def release(self) -> None:
        """Frees the graph, then the arena its outputs live in."""
        self.graph = None
        self.outputs = None
        self.arena = None


def run_host_batches(exec: Executor, fn, batches, outs) -> None:
    """Runs `fn(exec, *device_inputs) -> DeviceVec` over a sequence of host
    batches, with the copies overlapped: batch i + 1 uploads and batch i - 1
    downloads while the kernels of batch i run.

    `batches[i]` is a tuple of pinned host arrays (the same shapes and types
    for every batch); the result of batch i is copied into the pinned host
    array `outs[i]` (all of its elements, so `fn` should not leave a device
    length on it).  Uploads, kernels and downloads run on three streams of the
    executor's device, with two sets of device input buffers used in turn: a
    set is refilled only after the kernels that read it have finished.  The
    outputs of one call land in order on the download stream, so `outs` may
    repeat arrays (the last batch written wins).  Returns once every result
    is on the host; the executor is then bound to the caller's stream again.
    massively uploads, runs and downloads one batch at a time; this is for
    callers that stream many host batches through one device."""
    from .runtime import NP_TO_TORCH
    if not batches:
        return
    dev = exec.device
    caller = torch.cuda.current_stream(dev)
    up, comp, down = (torch.cuda.Stream(dev) for _ in range(3))
    slots = [[torch.empty(h.size, dtype=NP_TO_TORCH[h.dtype], device=f"cuda:{dev}")
              for h in batches[0]] for _ in range(2)]
    free = []
    for _ in range(2):
        e = torch.cuda.Event()
        e.record(caller)
        free.append(e)
    for s in (up, comp, down):
        s.wait_stream(caller)
    try:
        for i, batch in enumerate(batches):
            k = i % 2
            up.wait_event(free[k])
            with torch.cuda.stream(up):
                for t, h in zip(slots[k], batch):
                    if h.size != t.numel() or NP_TO_TORCH[h.dtype] != t.dtype:
                        raise ValueError("every batch has the first one's shapes and types")
                    src = torch.from_numpy(h.reshape(-1).view(np.uint8)).view(t.dtype)
                    t.copy_(src, non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(up)
            comp.wait_event(ready)
            with torch.cuda.stream(comp):
                exec.bind_current_stream()
                res = fn(exec, *[DeviceVec(exec, t) for t in slots[k]])
                done = torch.cuda.Event()
                done.record(comp)
            free[k] = done
            down.wait_event(done)
            with torch.cuda.stream(down):
                r = res.tensor
                dst = torch.from_numpy(outs[i].reshape(-1).view(np.uint8)).view(r.dtype)
                dst[:r.numel()].copy_(r, non_blocking=True)
                r.record_stream(down)
        down.synchronize()
    finally:
        with torch.cuda.stream(caller):
            exec.bind_current_stream()
        caller.wait_stream(down)
        caller.wait_stream(comp)
