"""Convergence of the smooth periodic advection configuration (rho = 1 + 0.2
sin 2 pi (x+y), u = v = 1, p = 1 to t = 0.5, SSP-RK3, Davis HLL, CFL <= 0.4):
the FP64 form's density L1 error against the exact cell averages falls with
the observed order log2(e(N/2)/e(N)) of the scheme, and the FP32-mixed form
stays on the FP64 curve down to its rounding floor.

Expected orders: WENO5 is fifth order in space, SSP-RK3 third order in time,
and at a fixed CFL dt ~ h, so the error tends to O(h^3) as N grows.  The
reference's WENO epsilon of 1e-2 (Weno5th.cpp:5, not the usual 1e-6) keeps the
weights near the linear ones on this smooth state, so the spatial error stays
fifth order and the combined order falls from about 5 towards 3 (the oracle at
N = 32, 64, 128: 5.6, 4.8, 3.8).  Asserted: order >= 2.8 between 128/256 and
256/512."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cfsb, workloads, n, prec):
    w = workloads.smooth_advection(n)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4)
    with cfsb.Solver(n, n, precision=cfsb.FP64, **kw) as s:
        s.set_state(w.U0)
        dt0 = s.compute_dt(w.cfl)
    nsteps = int(math.ceil(w.t_end / dt0))
    with cfsb.Solver(n, n, precision=prec, **kw) as s:
        s.set_state(w.U0)
        s.advance(nsteps, dt=w.t_end / nsteps)
        return s.get_state()


def test_observed_order_and_fp32_floor(cfsb, workloads):
    e64, e32, d = {}, {}, {}
    for n in (128, 256, 512):
        exact = workloads.smooth_advection_exact(n, 0.5)
        U64 = _run(cfsb, workloads, n, cfsb.FP64)
        U32 = _run(cfsb, workloads, n, cfsb.FP32_MIXED)
        e64[n] = float(np.abs(U64[0] - exact).mean())
        e32[n] = float(np.abs(U32[0] - exact).mean())
        d[n] = float(np.abs(U32[0] - U64[0]).mean())
    o1, o2 = math.log2(e64[128] / e64[256]), math.log2(e64[256] / e64[512])
    assert o1 >= 2.8 and o2 >= 2.8, (e64, o1, o2)
    assert e64[512] < 1e-9, e64
    # FP32-mixed: within its rounding floor of the FP64 solution
    for n in (128, 256, 512):
        assert d[n] <= 2e-6, (n, d)
        assert e32[n] <= e64[n] + 2e-6, (n, e32, e64)
