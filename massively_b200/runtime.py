"""Executor, device vectors and errors: the Python face of massively's runtime.

Mirrors massively/src/core/runtime.rs:22-389 (Executor, DeviceVec,
DeviceSlice) and massively/src/core/error.rs:5-14 (Error).  Device memory
is held in torch tensors (the caching allocator), the executor's C-ABI
handle enqueues every kernel on torch's current CUDA stream of its device,
and device-resident logical lengths (massively/src/core/extent.rs:17-36)
travel with the vectors that carry them.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np
import torch

from . import _native as N

# ------------------------------------------------------------------ errors --


class Error(Exception):
    """massively::Error (core/error.rs:5-14)."""

    code = N.LAUNCH

    def __eq__(self, other):
        return type(self) is type(other) and self.args == other.args

    def __hash__(self):
        return hash((type(self), self.args))


class LengthMismatch(Error):
    code = N.LENGTH_MISMATCH

    def __init__(self, left: int, right: int):
        super().__init__(left, right)
        self.left, self.right = left, right

    def __str__(self):
        return f"input lengths differ: {self.left} != {self.right}"


class OutputTooShort(Error):
    code = N.OUTPUT_TOO_SHORT

    def __init__(self, input: int, output: int):  # noqa: A002 - massively's field name
        super().__init__(input, output)
        self.input, self.output = input, output

    def __str__(self):
        return f"output length {self.output} is shorter than input length {self.input}"


class LengthTooLarge(Error):
    code = N.LENGTH_TOO_LARGE

    def __init__(self, len: int):  # noqa: A002
        super().__init__(len)
        self.len = len

    def __str__(self):
        return f"length does not fit in u32: {self.len}"


class InvalidSegmentation(Error):
    code = N.INVALID_SEGMENTATION

    def __str__(self):
        return "segmentation is not a valid ordered partition"


class UnboundColumn(Error):
    code = N.UNBOUND_COLUMN

    def __str__(self):
        return "column is not bound to device storage"


class ForeignExecutor(Error):
    code = N.FOREIGN_EXECUTOR

    def __str__(self):
        return "executor does not own this device data"


class Launch(Error):
    code = N.LAUNCH

    def __init__(self, message: str):
        super().__init__(message)
        self.message = message

    def __str__(self):
        return f"launch failed: {self.message}"


def check(status: int) -> None:
    """Raises the Error subclass of a non-zero C-ABI status."""
    if status == N.OK:
        return
    msg, left, right = N.last_error()
    if status == N.LENGTH_MISMATCH:
        raise LengthMismatch(left, right)
    if status == N.OUTPUT_TOO_SHORT:
        raise OutputTooShort(left, right)
    if status == N.LENGTH_TOO_LARGE:
        raise LengthTooLarge(left)
    if status == N.INVALID_SEGMENTATION:
        raise InvalidSegmentation()
    if status == N.UNBOUND_COLUMN:
        raise UnboundColumn()
    if status == N.FOREIGN_EXECUTOR:
        raise ForeignExecutor()
    raise Launch(msg)


# ------------------------------------------------------------------- types --

NP_TO_ID = {np.dtype(np.uint8): N.U8, np.dtype(np.uint16): N.U16, np.dtype(np.uint32): N.U32,
            np.dtype(np.uint64): N.U64, np.dtype(np.int8): N.I8, np.dtype(np.int16): N.I16,
            np.dtype(np.int32): N.I32, np.dtype(np.int64): N.I64,
            np.dtype(np.float32): N.F32, np.dtype(np.float64): N.F64}
ID_TO_NP = {v: k for k, v in NP_TO_ID.items()}
NP_TO_TORCH = {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
               np.dtype(np.uint32): torch.uint32, np.dtype(np.uint64): torch.uint64,
               np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16,
               np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
               np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}
TORCH_TO_NP = {v: k for k, v in NP_TO_TORCH.items()}

MINDEX_MAX = 0xFFFFFFFF


def value_bits(value, dtype) -> int:
    """Raw little-endian bits of one value of `dtype`, zero-extended to 64."""
    arr = np.array([value]).astype(np.dtype(dtype), copy=False) \
        if not isinstance(value, np.generic) else np.array([value], dtype=np.dtype(dtype))
    raw = arr.view(np.uint8)
    return int.from_bytes(raw.tobytes(), "little")


def scalar_buffer(value, dtype) -> C.Array:
    """An 8-byte host buffer holding one value of `dtype` (for init args)."""
    buf = (C.c_uint64 * 1)(value_bits(value, dtype))
    return buf


# ---------------------------------------------------------------- executor --

class Executor:
    """massively::Executor (core/runtime.rs:22-197): a device, its current
    CUDA stream and the library handle; `id` identifies owned storage."""

    def __init__(self, device: int = 0):
        self.device = int(device)
        self._lib = N.lib()
        h = C.c_void_p()
        check(self._lib.mb_executor_create(self.device, C.byref(h)))
        self._h = h
        self.id = int(self._lib.mb_executor_id(h))
        self._finalizer = weakref.finalize(self, self._lib.mb_executor_destroy, h)
        self.bind_current_stream()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def bind_current_stream(self) -> None:
        """Enqueue on torch's current stream of this device from now on."""
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream().cuda_stream
        check(self._lib.mb_set_stream(self._h, C.c_void_p(s)))

    def set_stream(self, stream: torch.cuda.Stream | None) -> None:
        """Enqueue on `stream` (a torch stream); None = the executor's own."""
        if stream is None:
            check(self._lib.mb_use_own_stream(self._h))
        else:
            check(self._lib.mb_set_stream(self._h, C.c_void_p(stream.cuda_stream)))

    def sync(self) -> None:
        """Executor::sync: waits and reports device-side failures."""
        check(self._lib.mb_sync(self._h))

    # -- storage -----------------------------------------------------------

    def alloc(self, dtype, n: int) -> "DeviceVec":
        """Executor::alloc: uninitialised device storage of `n` items."""
        if n > MINDEX_MAX:
            raise LengthTooLarge(n)
        return DeviceVec(self, self.storage(NP_TO_TORCH[np.dtype(dtype)], int(n)))

    def storage(self, tdtype: torch.dtype, n: int) -> torch.Tensor:
        """`n` items of device storage: a fresh tensor, or the next slice of
        the executor's arena while one is set (Arena)."""
        a = getattr(self, "_arena", None)
        if a is None:
            return torch.empty(n, dtype=tdtype, device=f"cuda:{self.device}")
        return a.take(tdtype, n, self.device)

    def zeros(self, dtype, n: int) -> "DeviceVec":
        v = self.alloc(dtype, n)
        v.tensor.zero_()
        return v

    def to_device(self, host) -> "DeviceVec":
        """Executor::to_device (runtime.rs:98-120)."""
        a = np.ascontiguousarray(np.asarray(host))
        if a.ndim != 1:
            a = a.reshape(-1)
        if a.size > MINDEX_MAX:
            raise LengthTooLarge(a.size)
        t = torch.from_numpy(a.view(np.uint8).copy()).view(NP_TO_TORCH[a.dtype]) if a.size else \
            torch.empty(0, dtype=NP_TO_TORCH[a.dtype])
        return DeviceVec(self, t.to(f"cuda:{self.device}"))

    def to_device_pinned(self, host: np.ndarray) -> "DeviceVec":
        """Stream-ordered upload of a host array living in pinned memory."""
        src = torch.from_numpy(host.reshape(-1).view(np.uint8)).view(NP_TO_TORCH[host.dtype])
        t = torch.empty(host.size, dtype=NP_TO_TORCH[host.dtype], device=f"cuda:{self.device}")
        t.copy_(src, non_blocking=True)
        return DeviceVec(self, t)

    def copy_to_pinned(self, vec: "DeviceVec", out: np.ndarray) -> int:
        """Downloads a vector (its logical length) into a pinned host array;
        returns the number of items written."""
        n = vec.logical_len()
        dst = torch.from_numpy(out.reshape(-1).view(np.uint8)).view(vec.tensor.dtype)
        dst[:n].copy_(vec.tensor[:n], non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return n

    def from_tensor(self, t: torch.Tensor) -> "DeviceVec":
        """Adopts a 1-D contiguous CUDA tensor as storage owned by this executor."""
        if not t.is_cuda or t.dim() != 1 or not t.is_contiguous():
            raise UnboundColumn()
        return DeviceVec(self, t)

    def to_host(self, vec) -> np.ndarray:
        """Executor::to_host (runtime.rs:146-177): honours a device length."""
        if not isinstance(vec, DeviceVec):
            raise UnboundColumn()
        if vec.owner != self.id:
            raise ForeignExecutor()
        n = vec.logical_len()
        out = vec.tensor[:n].cpu()
        return out.view(torch.uint8).numpy().view(vec.dtype) if n else np.empty(0, vec.dtype)

    def reserve_pool(self, nbytes: int) -> None:
        """Grows the device's stream-ordered pool to hold `nbytes` (capped
        at 90% of free memory) by allocating and freeing one block: later
        allocations up to that size reuse reserved memory instead of growing
        the pool in the middle of the work (a slow driver path)."""
        free, _ = torch.cuda.mem_get_info(self.device)
        n = int(min(nbytes, free * 0.9))
        if n <= 0:
            return
        with torch.cuda.device(self.device):
            t = torch.empty(n, dtype=torch.uint8, device=f"cuda:{self.device}")
            del t
            torch.cuda.synchronize(self.device)

    def pool_stats(self) -> tuple[int, int]:
        used, res = C.c_uint64(), C.c_uint64()
        check(self._lib.mb_pool_stats(self._h, C.byref(used), C.byref(res)))
        return int(used.value), int(res.value)


class Arena:
    """Storage for the calls made while it is set on an executor
    (`with arena.on(exec):`): in "record" mode allocations are ordinary
    tensors and only their sizes are noted; in "serve" mode they are
    consecutive 256-byte-aligned slices of one buffer allocated beforehand.
    A CUDA graph captured in "serve" mode (pipeline.Captured) therefore makes
    no allocation of torch's during capture: every buffer it reads or writes
    belongs to the arena, which lives exactly as long as its owner keeps it."""

    ALIGN = 256

    def __init__(self):
        self.sizes: list[int] = []
        self.buf: torch.Tensor | None = None
        self.off = 0

    @staticmethod
    def _round(nbytes: int) -> int:
        return (nbytes + Arena.ALIGN - 1) // Arena.ALIGN * Arena.ALIGN

    def allocate(self, device: int) -> None:
        """Switches from recording to serving: one buffer for the sizes
        recorded so far."""
        total = sum(self._round(s) for s in self.sizes)
        self.buf = torch.empty(max(total, self.ALIGN), dtype=torch.uint8, device=f"cuda:{device}")
        self.off = 0

    def take(self, tdtype: torch.dtype, n: int, device: int) -> torch.Tensor:
        nbytes = n * torch.empty(0, dtype=tdtype).element_size()
        if self.buf is None:
            self.sizes.append(nbytes)
            return torch.empty(n, dtype=tdtype, device=f"cuda:{device}")
        end = self.off + self._round(nbytes)
        if end > self.buf.numel():
            raise RuntimeError("arena exhausted: the calls allocate more than when recorded")
        t = self.buf[self.off:self.off + nbytes].view(tdtype)
        self.off = end
        return t

    class _On:
        def __init__(self, arena, exec):
            self.arena, self.exec = arena, exec

        def __enter__(self):
            self.prev = getattr(self.exec, "_arena", None)
            self.exec._arena = self.arena
            return self.arena

        def __exit__(self, *exc):
            self.exec._arena = self.prev
            return False

    def on(self, exec: "Executor"):
        return Arena._On(self, exec)


class DeviceVec:
    """massively::DeviceVec / DeviceSlice (runtime.rs:200-389): 1-D device
    storage owned by one executor, optionally with a device-resident logical
    length (LogicalExtent::Device)."""

    def __init__(self, exec: Executor, tensor: torch.Tensor, len_dev: torch.Tensor | None = None):
        self.owner = exec.id
        self.device = exec.device
        self.tensor = tensor
        self.len_dev = len_dev

    @property
    def dtype(self) -> np.dtype:
        return TORCH_TO_NP[self.tensor.dtype]

    @property
    def dtype_id(self) -> int:
        return NP_TO_ID[self.dtype]

    def __len__(self) -> int:
        return self.tensor.numel()

    def capacity(self) -> int:
        return self.tensor.numel()

    def logical_len(self) -> int:
        """The length on the host (reads the device length: a sync)."""
        if self.len_dev is None:
            return self.tensor.numel()
        return min(int(self.len_dev.cpu().item()), self.tensor.numel())

    def with_len_dev(self, len_dev: torch.Tensor) -> "DeviceVec":
        v = DeviceVec.__new__(DeviceVec)
        v.owner, v.device, v.tensor, v.len_dev = self.owner, self.device, self.tensor, len_dev
        return v

    def slice(self, start: int = 0, stop: int | None = None) -> "DeviceVec":
        """A zero-copy view of [start, stop) (DeviceSlice)."""
        n = self.tensor.numel()
        stop = n if stop is None else min(stop, n)
        v = DeviceVec.__new__(DeviceVec)
        v.owner, v.device, v.len_dev = self.owner, self.device, None
        v.tensor = self.tensor[start:stop]
        return v

    def data_ptr(self) -> int:
        return self.tensor.data_ptr()

    def to_src(self) -> N.mb_src:
        s = N.mb_src()
        s.kind = N.SRC_COLUMN
        s.dtype = s.vtype = self.dtype_id
        s.map = 0
        s.data = self.tensor.data_ptr() if self.tensor.numel() else None
        s.len = self.tensor.numel()
        s.owner = self.owner
        s.len_dev = self.len_dev.data_ptr() if self.len_dev is not None else None
        return s

    def to_col(self) -> N.mb_col:
        c = N.mb_col()
        c.data = self.tensor.data_ptr() if self.tensor.numel() else None
        c.dtype = self.dtype_id
        c.len = self.tensor.numel()
        c.owner = self.owner
        return c

    def __repr__(self):
        return f"DeviceVec(len={len(self)}, dtype={self.dtype}, owner={self.owner})"
