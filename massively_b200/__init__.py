"""massively_b200: B200-native primitives with massively's API.

    from massively_b200 import Executor, vector, seg, lazy, op, zip2
    exec = Executor(0)
    keys = exec.to_device(np.array([3, 1, 2], np.uint32))
    out = vector.radix_sort_by_key(exec, keys, exec.to_device(np.array([30, 10, 20], np.uint32)))

Every algorithm runs in hand-written sm_100a CUDA kernels of
libmassively_b200.so, reached through its C ABI (include/massively_b200.h);
there is no CPU fallback.

Device memory: DeviceVec storage comes from torch, the kernels' scratch from
the device's stream-ordered default pool.  When this package is imported
before torch and the process has not configured torch's allocator itself,
torch is pointed at that same pool (backend:cudaMallocAsync), so the two
never hold separate caches of freed memory (which, with several streams,
can leave one side out of memory while the other sits on free blocks).
torch reads that setting when it is imported, so it is left alone once
torch is loaded.
"""
import os as _os
import sys as _sys

if "torch" not in _sys.modules:
    _os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "backend:cudaMallocAsync")

from . import lazy, op, seg, vector  # noqa: E402,F401
from .iter import Zip, zip2, zip3, zip4, zip5, zip6, zip7, zip8, zip9, zip10, zip11, zip12  # noqa
from .runtime import (DeviceVec, Error, Executor, ForeignExecutor, InvalidSegmentation,  # noqa
                      Launch, LengthMismatch, LengthTooLarge, OutputTooShort, UnboundColumn)

MIndex = "uint32"
MFlag = "uint32"
