"""Failure detection without a GPU fault: the bounded waits of the persistent kernels.

The batch and server kernels wait on counters that other blocks advance; each wait gives up
after its time (or poll) bound, counts a timeout and raises an abort flag that ends every
block.  qcb_wait_selftest makes that happen on purpose (four blocks wait on a flag that
nothing sets) and the test checks the status words, the elapsed time, and that the context
still runs the heatbath afterwards.
"""
import ctypes as C
import time

import numpy as np
import pytest

import oracle as orc
import qcb
from qcb import _lib

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_stays_usable(ctx):
    lib = _lib.lib()
    t, a = C.c_uint32(), C.c_uint32()
    t0 = time.perf_counter()
    _lib.check(lib.qcb_wait_selftest(ctx.h, 0.25, C.byref(t), C.byref(a)))
    dt = time.perf_counter() - t0
    assert t.value == 1 and a.value == 1
    assert 0.2 < dt < 5.0
    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 77)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    _lib.check(lib.qcb_heatbath(f.h, 6.0, 1, 1, 5, 0))
    ref, _ = orc.heatbath_cb(u, dims, 6.0, 1, 1, 5, 0)
    assert np.abs(f.get_links() - ref).max() < 1e-11
    f.close()


def test_wait_selftest_rejects_bad_limits(ctx):
    lib = _lib.lib()
    t, a = C.c_uint32(), C.c_uint32()
    assert lib.qcb_wait_selftest(ctx.h, 0.0, C.byref(t), C.byref(a)) == 1
    assert lib.qcb_wait_selftest(ctx.h, 60.0, C.byref(t), C.byref(a)) == 1
    assert lib.qcb_wait_selftest(None, 0.1, C.byref(t), C.byref(a)) == 1
