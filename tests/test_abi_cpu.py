"""C-ABI checks that need no GPU: the library loads, exports every symbol
the header declares, and argument errors map onto massively's Error variants
without touching a device."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "massively_b200.h")


def _declared():
    return sorted(set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", open(HEADER).read())))


def test_library_exports_every_declared_symbol():
    from massively_b200 import _native
    lib = _native.lib()
    missing = [s for s in _declared() if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.mb_abi_version() == 1


def test_header_compiles_as_c():
    # The boundary is plain C: the header must compile with a C compiler.
    src = '#include "massively_b200.h"\nint main(void) { mb_src s; mb_col c; (void)s; (void)c; ' \
          'return MB_OK; }\n'
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only",
                        f"-I{os.path.dirname(HEADER)}", "-x", "c", "-"], input=src, text=True,
                       capture_output=True)
    assert r.returncode == 0, r.stderr


def test_struct_layouts_match_ctypes():
    from massively_b200 import _native as N
    assert C.sizeof(N.mb_src) == 72
    assert C.sizeof(N.mb_col) == 32
    assert C.sizeof(N.mb_error_detail) == 16


def test_null_executor_is_an_error_not_a_crash():
    from massively_b200 import _native as N
    lib = N.lib()
    assert lib.mb_sync(None) == N.LAUNCH
    assert b"null executor" in lib.mb_last_error_message()
    assert lib.mb_tune_config_count(1) >= 1
    assert lib.mb_tune_describe(1, 0)


def test_error_classes_mirror_massively():
    import massively_b200 as mb
    assert mb.LengthMismatch(2, 1) == mb.LengthMismatch(2, 1)
    assert str(mb.LengthMismatch(2, 1)) == "input lengths differ: 2 != 1"
    assert str(mb.OutputTooShort(5, 3)) == "output length 3 is shorter than input length 5"
    assert str(mb.InvalidSegmentation()) == "segmentation is not a valid ordered partition"
    assert str(mb.ForeignExecutor()) == "executor does not own this device data"


def test_zip_rejects_ragged_columns():
    import numpy as np

    import massively_b200 as mb

    class Col:
        def __init__(self, n):
            self.n = n
            self.dtype = np.dtype(np.uint32)

        def __len__(self):
            return self.n

    with pytest.raises(mb.LengthMismatch):
        mb.zip2(Col(3), Col(4))
    z = mb.zip3(Col(5), Col(5), Col(5))
    assert len(z) == 5 and len(z.into_columns()) == 3
