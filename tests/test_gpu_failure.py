"""Failure detection on the GPU without a fault: a bounded wait made to run
out (an mbarrier nothing arrives on) reports the timeout to the host and the
kernel returns; the same context then searches normally."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(golden):
    import liteqg_b200
    from liteqg_b200._capi import lib

    L = lib()
    out = C.c_uint32(7)
    assert L.lqg_selftest_bounded_wait(0, 256, C.byref(out)) == 0, L.lqg_last_error()
    assert out.value == 1
    assert L.lqg_selftest_bounded_wait(0, 0, C.byref(out)) == 1  # argument check
    g = golden["u48"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    ix.set_ef(50)
    assert np.array_equal(ix.search(g["queries"], 10), g["expected"][(50, 10)])
