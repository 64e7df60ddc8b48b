"""A run continued from a snapshot in a new context takes the same steps, bit
for bit, as the uninterrupted run (FP32-mixed: stochastic rounding hashed with
the step counter, storage offsets, the CFL maximum carried between advance
calls).  The reference only writes snapshots (Output.cpp:20), so a restart is
this engine's addition; a restart from the state alone is a different run."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
def test_resume_from_snapshot_is_bit_exact(cfsb, workloads, tmp_path, prec):
    snapshot = importlib.import_module("2d_compressible_flow_solver_b200.snapshot")
    w = workloads.riemann_quadrants(96, 80, seed=5)
    kw = dict(precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4)
    with cfsb.Solver(96, 80, **kw) as s:
        s.set_state(w.U0)
        s.advance(10, cfl=0.5)
        ref = s.get_state()
    with cfsb.Solver(96, 80, **kw) as s:
        s.set_state(w.U0)
        t, dt = s.advance(5, cfl=0.5)
        path = snapshot.write_solver_snapshot(s, tmp_path / "snap", time=t, dt=dt, fmt="raw")
    run = snapshot.read_run(path)
    assert run["step"] == 5 and run["cfl_max"] > 0 and run["time"] == t and run["dt"] == dt
    with cfsb.Solver(96, 80, **kw) as s:
        snapshot.resume_solver(s, path)
        assert s.run_counters()["step"] == 5
        s.advance(5, cfl=0.5)
        got = s.get_state()
    assert np.array_equal(got, ref)
    if prec == cfsb.FP32_MIXED:
        # the state alone (offsets from its own means, step 0, a fresh CFL
        # reduction) continues a different run
        d = snapshot.read_snapshot(path)
        with cfsb.Solver(96, 80, **kw) as s:
            s.set_state(np.stack([d["Rho"], d["Mu"], d["Mv"], d["Energy"]]))
            s.advance(5, cfl=0.5)
            assert not np.array_equal(s.get_state(), ref)


def test_set_step_is_refused_inside_a_step(cfsb, workloads):
    w = workloads.riemann_quadrants(32, 32, seed=1)
    with cfsb.Solver(32, 32) as s:
        s.set_state(w.U0)
        s.stage(1, 1e-4)
        with pytest.raises(cfsb.CfsError) as e:
            s._check(s._lib.cfs_set_step(s._ctx, 3, 0.0))
        assert e.value.code == 4


def _with_nan_cell(U):
    U = U.copy()
    U[0, U.shape[1] // 2, U.shape[2] // 3] = np.nan
    return U


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_a_non_finite_fluid_cell_is_reported(cfsb, workloads, prec):
    """One NaN cell in the state (a host input, no device fault): the CFL
    reduction reports it (CFS_ERR_NUMERIC) instead of skipping the cell."""
    w = workloads.riemann_quadrants(64, 48, seed=2)
    with cfsb.Solver(64, 48, precision=prec) as s:
        s.set_state(_with_nan_cell(w.U0))
        with pytest.raises(cfsb.CfsError) as e:
            s.compute_dt(0.5)
        assert e.value.code == 5
        with pytest.raises(cfsb.CfsError) as e:
            s.advance(2, cfl=0.5)
        assert e.value.code == 5


@pytest.mark.parametrize("prec", [0, 1])
def test_a_blow_up_during_an_advance_is_reported(cfsb, workloads, prec):
    """The reference's scheme (no positivity fallback) reaches NaN behind a
    Mach-3 cylinder within its first steps (as the oracle does); the advance
    that produces it returns CFS_ERR_NUMERIC instead of stepping on with a
    finite dt taken over the remaining cells."""
    w = workloads.mach3_cylinder(128, 64)
    with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=w.bc,
                     bc_prim=w.bc_prim) as s:
        s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP)
        s.set_state(w.U0)
        with pytest.raises(cfsb.CfsError) as e:
            s.advance(6, cfl=0.5)
        assert e.value.code == 5
