"""Every stage-kernel variant (rows x warps x occupancy x load schedule,
cfs_variant_info) computes the same stage: against variant 1, relative
L-infinity <= 1e-12 in FP64 and <= 1e-5 in FP32-mixed after 6 steps (the
variants are separate compilations, so FMA contraction may differ in the last
bits).  Cases: four-quadrant Riemann problem with transmissive sides, and a
cylinder with the slip-wall IB and the body positivity fallback."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cfsb, w, prec, variant, circle=None):
    with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=w.bc,
                     bc_prim=w.bc_prim, variant=variant,
                     positivity=cfsb.POSITIVITY_BODY if circle else cfsb.POSITIVITY_OFF) as s:
        if circle:
            s.build_circle(*circle, 400, cfsb.IB_BILINEAR_SLIP)
        s.set_state(w.U0)
        s.advance(6, dt=5e-4)
        return s.get_state()


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_variants_agree(cfsb, workloads, prec, tol):
    quad = workloads.riemann_quadrants(150, 130, seed=9)
    cyl = workloads.mach3_cylinder(192, 96)
    nvar = len(cfsb.variants())
    assert nvar >= 20
    for w, circle in ((quad, None), (cyl, cyl.circle)):
        ref = _run(cfsb, w, prec, 1, circle)
        assert np.all(np.isfinite(ref))
        scale = np.abs(ref).max()
        for v in range(2, nvar + 1):
            got = _run(cfsb, w, prec, v, circle)
            err = np.abs(got - ref).max() / scale
            assert err <= tol, (w.name, v, cfsb.variants()[v - 1], err)
