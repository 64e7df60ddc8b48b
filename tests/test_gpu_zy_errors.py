"""A failed device allocation is reported to its caller and does not fail the
calls that follow: the runtime records the failure as the thread's last CUDA
error too, which the library consumes when it reports the error, so the
launch checks of later calls do not report it again as their own."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_failed_allocation_leaves_later_calls_working(cfsb, workloads):
    w = workloads.smooth_advection(64)
    kw = dict(precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(2, 2, 2, 2))
    with cfsb.Solver(64, 64, **kw) as s:
        s.set_state(w.U0)
        s.advance(2, dt=1e-3)
        ref = s.get_state()
        # 2^31 - 1 faces ask for 412 GB of stencils: the first device allocation
        # fails and the call returns before any host buffer is read
        small = np.zeros(24)
        dp = ctypes.POINTER(ctypes.c_double)
        ptr = small.ctypes.data_as(dp)
        rc = s._lib.cfs_weno5_faces(s._ctx, 2**31 - 1, ptr, ptr, ptr)
        assert rc != 0
        msg = s._lib.cfs_last_error(s._ctx).decode().lower()
        assert "alloc" in msg or "memory" in msg, msg
        # the same context, and a new one, still run
        s.set_state(w.U0)
        s.advance(2, dt=1e-3)
        assert np.array_equal(s.get_state(), ref)
    with cfsb.Solver(64, 64, **kw) as s2:
        s2.set_state(w.U0)
        s2.advance(2, dt=1e-3)
        assert np.array_equal(s2.get_state(), ref)
