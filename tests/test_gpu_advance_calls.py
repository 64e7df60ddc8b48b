"""cfs_advance with a CFL step: K calls of one step take exactly the steps one
call of K steps takes (the CFL maximum of the state carries from one call's
last stage to the next call), in both throughput forms, on a periodic and on a
transmissive grid with a cylinder; a cfs_set_state in between starts afresh."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("case", ["periodic", "cylinder"])
def test_k_single_steps_equal_one_k_step_call(cfsb, workloads, prec, case):
    if case == "periodic":
        w = workloads.riemann_quadrants(96, 80, seed=4)
        kw = dict(bc=(cfsb.BC_PERIODIC,) * 4)
        body = None
    else:
        w = workloads.mach3_cylinder(192, 96)
        kw = dict(bc=w.bc, bc_prim=w.bc_prim, positivity=cfsb.POSITIVITY_FLOOR)
        body = w.circle
    runs = []
    for split in (False, True):
        with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, **kw) as s:
            if body:
                s.build_circle(*body, 400, cfsb.IB_BILINEAR_SLIP)
            s.set_state(w.U0)
            if split:
                t, last = 0.0, None
                for _ in range(7):
                    dt_t, last = s.advance(1, cfl=0.5)
                    t += dt_t
            else:
                t, last = s.advance(7, cfl=0.5)
            runs.append((t, last, s.get_state()))
    (t0, d0, U0), (t1, d1, U1) = runs
    assert t0 == t1 and d0 == d1
    assert np.array_equal(U0, U1)


def test_set_state_starts_the_cfl_afresh(cfsb, workloads):
    w = workloads.riemann_quadrants(64, 64, seed=5)
    with cfsb.Solver(64, 64, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4) as s:
        s.set_state(w.U0)
        s.advance(3, cfl=0.5)
        s.set_state(w.U0)          # back to the initial state: its own CFL maximum
        t_again = s.advance(1, cfl=0.5)[0]
    with cfsb.Solver(64, 64, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4) as s:
        s.set_state(w.U0)
        t_first = s.advance(1, cfl=0.5)[0]
    assert t_again == t_first
