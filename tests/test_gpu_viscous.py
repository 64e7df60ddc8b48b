"""Navier-Stokes (viscous) terms on the GPU against the C oracle's restatement
(oracle/cfs_oracle.c add_ns_terms), per RK step from the same state:
relative L-infinity <= 1e-12 for the FP64 form, <= 2e-5 for FP32-mixed."""
import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

MACH3 = (1.4, 3.0, 0.0, 1.0)


def _rel_linf(a, b):
    return max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(4))


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 2e-5)])
@pytest.mark.parametrize("bc", [(2, 2, 2, 2), (0, 0, 1, 0)])
@pytest.mark.parametrize("shape", [(72, 64), (53, 45)])  # 53 x 45: partial tiles in both directions
def test_navier_stokes_step_matches_oracle(cfsb, workloads, prec, tol, bc, shape):
    nx, ny = shape
    mu = 2e-3
    if bc == (2, 2, 2, 2):
        U = workloads.shear_layer(max(nx, ny), seed=2).U0[:, :nx, :ny].copy()
    else:
        U = workloads.riemann_quadrants(nx, ny, seed=6).U0
    cfg = ob.make_orc_config(nx, ny, rk=2, hll=1, bc=bc, bc_prim=[MACH3] * 4, viscous=1, mu=mu, prandtl=0.72,
                             mach=1.0)
    worst = 0.0
    with cfsb.Solver(nx, ny, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=bc, bc_prim=[MACH3] * 4,
                     viscous=cfsb.VISCOUS_NS, mu=mu, prandtl=0.72, mach=1.0) as s:
        for _ in range(5):
            dt = ob.orc_cfl_dt(cfg, U, 0.4)
            s.set_state(U)
            s.step(dt)
            got = s.get_state()
            ref, _ = ob.orc_run(cfg, U, 1, 3, dt=dt)
            worst = max(worst, _rel_linf(got, ref))
            U = ref
    assert worst <= tol, worst


def test_viscous_terms_change_the_solution(cfsb, workloads):
    """The viscous contribution is actually applied (inviscid and viscous runs differ
    by about mu * dt * second derivatives)."""
    n = 64
    U = workloads.shear_layer(n, seed=1).U0
    out = []
    for visc in (cfsb.VISCOUS_OFF, cfsb.VISCOUS_NS):
        with cfsb.Solver(n, n, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(2, 2, 2, 2), viscous=visc, mu=5e-3) as s:
            s.set_state(U)
            s.advance(4, cfl=0.4)
            out.append(s.get_state())
    assert np.abs(out[0][1] - out[1][1]).max() > 1e-6
