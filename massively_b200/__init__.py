"""massively_b200: B200-native primitives with massively's API.

    from massively_b200 import Executor, vector, seg, lazy, op, zip2
    exec = Executor(0)
    keys = exec.to_device(np.array([3, 1, 2], np.uint32))
    out = vector.radix_sort_by_key(exec, keys, exec.to_device(np.array([30, 10, 20], np.uint32)))

Every algorithm runs in hand-written sm_100a CUDA kernels of
libmassively_b200.so, reached through its C ABI (include/massively_b200.h);
there is no CPU fallback.
"""
from . import lazy, op, seg, vector  # noqa: F401
from .iter import Zip, zip2, zip3, zip4, zip5, zip6, zip7, zip8, zip9, zip10, zip11, zip12  # noqa
from .runtime import (DeviceVec, Error, Executor, ForeignExecutor, InvalidSegmentation,  # noqa
                      Launch, LengthMismatch, LengthTooLarge, OutputTooShort, UnboundColumn)

MIndex = "uint32"
MFlag = "uint32"
