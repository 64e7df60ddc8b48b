"""FP32-mixed storage rounding modes (cfg.rounding).

CFS_ROUND_STOCHASTIC rounds the state that ends each RK step stochastically
and the intermediate stage states to nearest; CFS_ROUND_STOCHASTIC_ALL rounds
every stage stochastically.  The increments of a stage are differences of FP32
fluxes and so lie on a coarse lattice; rounding them to nearest onto the
stored spacing does not average out, and the intermediate stages then carry
a small mass bias per step that depends on dt.  Stochastic rounding in every
stage has none: its mass drift is a random walk.  Both modes hash their random
bits from (cell, step, stage), so runs repeat bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cfsb, w, rounding, nsteps, dt):
    with cfsb.Solver(w.nx, w.ny, precision=cfsb.FP32_MIXED, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4, rounding=rounding) as s:
        s.set_state(w.U0)
        m0 = s.totals()
        s.advance(nsteps, dt=dt)
        return s.get_state(), (s.totals() - m0) / np.abs(m0)


def test_stochastic_all_repeats_and_conserves(cfsb, workloads):
    w = workloads.smooth_advection(256)
    with cfsb.Solver(256, 256, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4) as s:
        s.set_state(w.U0)
        dt = s.compute_dt(0.4)
        s.advance(1500, dt=dt)
        ref = s.get_state()
    a, drift_a = _run(cfsb, w, cfsb.ROUND_STOCHASTIC_ALL, 1500, dt)
    b, _ = _run(cfsb, w, cfsb.ROUND_STOCHASTIC_ALL, 1500, dt)
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a))
    # a random walk of 256^2 cells x 4,500 stage roundings of about 1e-8 each
    # stays near 1e-9 of the mass; the round-to-nearest bias of the
    # intermediate stages is of order 1e-11 per step
    assert abs(drift_a[0]) < 5e-9 and abs(drift_a[3]) < 5e-9, drift_a
    assert np.abs(a[0] - ref[0]).mean() < 1e-5
    # the modes differ (the intermediate stages round differently)
    c, _ = _run(cfsb, w, cfsb.ROUND_STOCHASTIC, 1500, dt)
    assert not np.array_equal(a, c)
    assert np.abs(c[0] - ref[0]).mean() < 1e-5


def test_unknown_rounding_mode_is_refused(cfsb):
    with pytest.raises(cfsb.CfsError):
        cfsb.Solver(64, 64, precision=cfsb.FP32_MIXED, rounding=3)
