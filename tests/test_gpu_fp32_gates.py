"""FP32-mixed error gates on the shocked configurations, every comparison on
one time-step sequence (the FP64 run's CFL steps, replayed as fixed steps).

On the four-quadrant configuration with the reference's own scheme the FP64
run is itself sensitive to rounding: perturbing its initial state by the FP32
unit roundoff (2^-24 per value, random signs) moves its density at t_end by
about as much as FP32 storage does.  The gate there is relative to that
sensitivity, measured in the same test.  On the uneven batch (Davis HLL,
SSP-RK3, floors) the four-quadrant cases meet the 1e-5 density L1 bound
directly; the cylinders' wakes amplify any difference over the run, so they
are held to finite, positive states and a looser bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_quadrant_configuration_fp32_within_fp64_sensitivity(cfsb, workloads):
    w = workloads.riemann_quadrants(256, 256, seed=1)
    kw = dict(rk=cfsb.RK_TVD3_REFERENCE, hll=cfsb.HLL_REFERENCE)
    with cfsb.Solver(256, 256, precision=cfsb.FP64, **kw) as s:
        s.set_state(w.U0)
        dts = [s.advance(1, cfl=0.5)[1] for _ in range(200)]
        U64 = s.get_state()

    def replay(prec, U0):
        with cfsb.Solver(256, 256, precision=prec, **kw) as s:
            s.set_state(U0)
            for dt in dts:
                s.advance(1, dt=dt)
            return s.get_state()

    U32 = replay(cfsb.FP32_MIXED, w.U0)
    sign = np.random.default_rng(7).choice([-1.0, 1.0], size=w.U0.shape)
    Up = replay(cfsb.FP64, w.U0 * (1.0 + sign * 2.0 ** -24))
    assert np.all(np.isfinite(U32)) and np.all(np.isfinite(Up))
    e32 = float(np.abs(U32[0] - U64[0]).mean())
    sens = float(np.abs(Up[0] - U64[0]).mean())
    # measured on a B200: FP32 1.2e-3, the FP64 run's own sensitivity 1.9e-3
    assert sens > 0
    assert e32 <= 3.0 * sens, (e32, sens)
    assert e32 < 1e-2, e32


def test_uneven_batch_fp32_against_fp64_per_case(cfsb, workloads):
    cases, states = workloads.batch_cases(48, seed=11, sizes=[64, 96, 128, 192, 256])
    kw = dict(positivity=cfsb.POSITIVITY_FLOOR)
    with cfsb.Batch(cases, precision=cfsb.FP64, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        seq = []
        for _ in range(200):
            b.advance(1, cfl=0.5)
            seq.append(b.dt_last())
        U64 = [b.get_state(k) for k in range(len(cases))]
    with cfsb.Batch(cases, precision=cfsb.FP32_MIXED, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        for d in seq:
            b.advance(1, dt=d)
        U32 = [b.get_state(k) for k in range(len(cases))]
    err = np.array([np.abs(a[0] - b_[0]).mean() for a, b_ in zip(U32, U64)])
    assert all(np.all(np.isfinite(U)) and U[0].min() > 0 for U in U32)
    quads = np.array(["circle" not in c for c in cases])
    # measured over 500 steps of the 512-case batch: four-quadrant cases at
    # most 2.4e-6, median of all cases 6e-7, cylinders at most 8.1e-5
    assert err[quads].max() <= 1e-5, err[quads].max()
    assert np.median(err) <= 5e-6, np.median(err)
    assert err[~quads].max() <= 1e-3, err[~quads].max()
