"""Every stage-kernel variant (rows x warps x occupancy x load schedule,
cfs_variant_info) computes the same stage: against variant 1, relative
L-infinity <= 1e-12 in FP64 and <= 1e-5 in FP32-mixed after 6 steps (the
variants are separate compilations, so FMA contraction may differ in the last
bits).  Cases cover the row march's feature sets: a periodic four-quadrant
problem (no edge code), the same with the face positivity fallback and the RHS
copy, the four-quadrant problem with transmissive sides (boundary-face fluxes),
and a cylinder with the slip-wall IB and the body positivity fallback (cell
flags).  The feature sets themselves agree where they must: all-fluid cell
types, and a positivity fallback that never triggers, change nothing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cfsb, w, prec, variant, circle=None, bc=None, positivity=None, keep_rhs=False, types=None):
    if positivity is None:
        positivity = cfsb.POSITIVITY_BODY if circle else cfsb.POSITIVITY_OFF
    with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=w.bc if bc is None else bc, bc_prim=w.bc_prim, variant=variant, positivity=positivity,
                     keep_rhs=keep_rhs) as s:
        if circle:
            s.build_circle(*circle, 400, cfsb.IB_BILINEAR_SLIP)
        if types is not None:
            s.set_cell_types(types)
        s.set_state(w.U0)
        s.advance(6, dt=5e-4)
        return s.get_state()


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_variants_agree(cfsb, workloads, prec, tol):
    quad = workloads.riemann_quadrants(150, 130, seed=9)
    cyl = workloads.mach3_cylinder(192, 96)
    nvar = len(cfsb.variants())
    assert nvar >= 10
    per = (cfsb.BC_PERIODIC,) * 4
    cases = [("periodic", quad, {"bc": per}),
             ("periodic+face+rhs", quad, {"bc": per, "positivity": cfsb.POSITIVITY_FACE, "keep_rhs": True}),
             ("transmissive", quad, {}),
             ("cylinder", cyl, {"circle": cyl.circle})]
    for name, w, kw in cases:
        ref = _run(cfsb, w, prec, 1, **kw)
        assert np.all(np.isfinite(ref))
        scale = np.abs(ref).max()
        for v in range(2, nvar + 1):
            got = _run(cfsb, w, prec, v, **kw)
            err = np.abs(got - ref).max() / scale
            assert err <= tol, (name, v, cfsb.variants()[v - 1], err)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_feature_sets_agree(cfsb, workloads, prec, tol):
    w = workloads.smooth_advection(96)
    per = (cfsb.BC_PERIODIC,) * 4
    ref = _run(cfsb, w, prec, 0, bc=per)
    scale = np.abs(ref).max()
    for kw in ({"types": np.zeros((w.nx, w.ny), np.uint8)},
               {"positivity": cfsb.POSITIVITY_FACE},
               {"positivity": cfsb.POSITIVITY_FLOOR, "types": np.zeros((w.nx, w.ny), np.uint8)},
               {"keep_rhs": True}):
        got = _run(cfsb, w, prec, 0, bc=per, **kw)
        err = np.abs(got - ref).max() / scale
        assert err <= tol, (kw.keys(), err)


@pytest.mark.parametrize("prec", [0, 1])
def test_row_chunk_changes_no_bit(cfsb, workloads, prec):
    """cfs_config.march_rows (rows of one warp's work item; 0 = chosen per
    launch to fill whole waves): a chunk boundary only repeats the x-flux of
    the face between two chunks in both, with the same arithmetic, so every
    chunk gives the same state bit for bit, on a grid whose rows the chunks do
    not divide, with transmissive sides and with a cylinder."""
    quad = workloads.riemann_quadrants(150, 130, seed=9)
    cyl = workloads.mach3_cylinder(192, 96)
    for w, circle in ((quad, None), (cyl, cyl.circle)):
        outs = []
        for rows in (0, 1, 7, 32, 61, 500):
            with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                             bc=w.bc, bc_prim=w.bc_prim, march_rows=rows,
                             positivity=cfsb.POSITIVITY_BODY if circle else cfsb.POSITIVITY_OFF) as s:
                if circle:
                    s.build_circle(*circle, 400, cfsb.IB_BILINEAR_SLIP)
                s.set_state(w.U0)
                t, _ = s.advance(4, cfl=0.5)
                outs.append((s.get_state(), t))
        assert np.all(np.isfinite(outs[0][0]))
        for got, t in outs[1:]:
            assert np.array_equal(got, outs[0][0])
            assert t == outs[0][1]


def test_row_chunk_out_of_range_is_refused(cfsb):
    with pytest.raises(cfsb.CfsError):
        cfsb.Solver(64, 64, march_rows=-1)
    with pytest.raises(cfsb.CfsError):
        cfsb.Solver(64, 64, march_rows=4097)
