"""Failure detection without a GPU fault: every spin-wait of the library is
bounded (2 s of %globaltimer), after which the kernel records the failure
in the executor's status word, sets the launch's abort word so its other
waiting blocks stop too, and returns.  mb_check_bounded_waits runs the
library's own waits against a condition that never comes (a look-back
predecessor that never publishes; an mbarrier whose bulk-copy bytes never
arrive); the test checks that the launch ends, that mb_sync reports
Launch{message} once, and that the executor keeps working afterwards."""
import time

import numpy as np
import pytest

from tests.gpu_util import executor, gpu, seeded

pytestmark = gpu


@pytest.fixture(scope="module")
def ex():
    return executor()


@pytest.mark.parametrize("kind", [0, 1], ids=["lookback", "mbarrier"])
def test_bounded_wait_gives_up_and_reports_launch(ex, kind, orc):
    import massively_b200 as mb
    from massively_b200 import _native as N
    from massively_b200 import vector
    from massively_b200.runtime import Launch, check
    ex.sync()
    t0 = time.perf_counter()
    check(N.lib().mb_check_bounded_waits(ex.handle, kind))
    with pytest.raises(Launch) as e:
        ex.sync()
    waited = time.perf_counter() - t0
    assert "look-back" in str(e.value)
    assert 1.5 < waited < 30.0, f"the wait ended after {waited:.2f} s"
    ex.sync()  # reported once, then cleared
    # the context is still usable: a sort right after is exact
    keys = seeded(np.uint32, 100_000, 13)
    sk, sv = vector.radix_sort_pairs(ex, ex.to_device(keys),
                                     ex.to_device(np.arange(keys.size, dtype=np.uint32)))
    perm = orc.radix_perm([keys])
    np.testing.assert_array_equal(ex.to_host(sv), perm)
    ex.sync()
    assert isinstance(ex, mb.Executor)


def test_unknown_check_is_an_error(ex):
    from massively_b200 import _native as N
    assert N.lib().mb_check_bounded_waits(ex.handle, 7) == N.LAUNCH
