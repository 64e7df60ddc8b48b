"""GPU parity of the stage engine, through the C ABI (ctypes binding), against
the reference's own outputs (golden fixtures) and the C oracle.

Tolerances:
  * CFS_FP64_EXACT: bit-identical (reference operation order, no FMA).
  * CFS_FP64: relative L-infinity <= 1e-12 per RK step, each step started from
    the same state on both sides (relative = max|diff| / max|U| per variable).
  * CFS_FP32_MIXED: density L1 error <= 1e-5 against the FP64 path at t_end,
    conservation drift <= 1e-6 relative.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
MACH3 = (1.4, 3.0, 0.0, 1.0)


def _load(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def _rel_linf(a, b):
    out = 0.0
    for v in range(4):
        scale = max(np.abs(b[v]).max(), 1e-300)
        out = max(out, np.abs(a[v] - b[v]).max() / scale)
    return out


def run_counters(s, first, count, cfl=0.0, dt=0.0, stages_per_step=3):
    """Drives the engine like Run::solver's loop: counters first..first+count-1,
    CFL dt recomputed at each step's first stage."""
    dts = []
    for k in range(first, first + count):
        is_start = (k % stages_per_step) == 1 if stages_per_step == 3 else (k % 2) == 1
        if cfl > 0 and is_start:
            dt = s.compute_dt(cfl)
        dts.append(dt)
        s.stage(k, dt)
    return np.array(dts)


# ---------------------------------------------------------------- unit level
def test_weno_and_hll_exact_are_bitwise_the_reference(cfsb):
    g = _load("faces_weno_hll")
    with cfsb.Solver(8, 8, precision=cfsb.FP64_EXACT) as s:
        left, right = s.weno5_faces(g["stencils"])
        assert np.array_equal(left, g["left"])
        assert np.array_equal(right, g["right"])
        for d in range(2):
            assert np.array_equal(s.hll_faces(d, g["L"], g["R"]), g["F"][d])


@pytest.mark.parametrize("prec,tol", [(1, 2e-5), (0, 1e-13)])
def test_weno_and_hll_fast_forms(cfsb, prec, tol):
    g = _load("faces_weno_hll")
    with cfsb.Solver(8, 8, precision=prec) as s:
        left, right = s.weno5_faces(g["stencils"])
        scale = np.abs(g["left"]).max(axis=0)
        assert np.all(np.abs(left - g["left"]) <= tol * scale * 10)
        assert np.all(np.abs(right - g["right"]) <= tol * scale * 10)
        for d in range(2):
            F = s.hll_faces(d, g["L"], g["R"])
            ok = np.isfinite(g["F"][d])
            fs = np.abs(g["F"][d][ok]).max()
            assert np.all(np.abs(F[ok] - g["F"][d][ok]) <= tol * fs * 10)


# ------------------------------------------------------ stage, exact form
@pytest.mark.parametrize("name", ["quadrants_tvd3_48x40_cfl", "quadrants_tvd2_32x32_cfl",
                                  "quadrants_dirichlet_tvd3_40x32"])
def test_exact_stage_reproduces_reference_fixture(cfsb, name):
    g = _load(name)
    nx, ny, nst = int(g["cfg_nx"]), int(g["cfg_ny"]), int(g["cfg_nstages"])
    integ = int(g["cfg_integrator"])
    bc = tuple(int(b) for b in g.get("cfg_bc", np.zeros(4)))
    bc_prim = g["cfg_bc_prim"] if "cfg_bc_prim" in g else None
    rk = cfsb.RK_TVD2 if integ == 2 else cfsb.RK_TVD3_REFERENCE
    with cfsb.Solver(nx, ny, precision=cfsb.FP64_EXACT, rk=rk, bc=bc, bc_prim=bc_prim, keep_rhs=True) as s:
        s.set_state(g["U0"])
        dts = run_counters(s, 1, nst, cfl=float(g.get("cfg_cfl", 0.0)), dt=float(g.get("cfg_dt", 1e-3)),
                           stages_per_step=2 if integ == 2 else 3)
        assert np.array_equal(dts, g["dt"])
        assert np.array_equal(s.get_state(), g["U"])
        assert np.array_equal(s.get_rhs(), g["rhs"])


def test_exact_stage_with_immersed_circle_reproduces_reference_fixture(cfsb):
    g = _load("circle_tvd3_64x64")
    lst = _load("circle_64x64_lists")
    with cfsb.Solver(64, 64, precision=cfsb.FP64_EXACT, bc=(1, 0, 0, 0), bc_prim=[MACH3] * 4) as s:
        s.build_circle(0.2, 0.45, 0.55, 400, cfsb.IB_REFERENCE)
        types, cells, donors, images = s.get_ib()
        assert np.array_equal(types, lst["types"]) and np.array_equal(cells, lst["cells"])
        assert np.array_equal(donors, lst["donors"]) and np.array_equal(images, lst["images"])
        s.set_state(g["U0"])
        run_counters(s, 1, int(g["cfg_nstages"]), dt=float(g["cfg_dt"]))
        assert np.array_equal(s.get_state(), g["U"], equal_nan=True)


def test_exact_long_run_matches_oracle(cfsb, workloads):
    """Quadrant Riemann state, 128^2, TVD3 as written, CFL 0.5, 60 steps."""
    nx = ny = 128
    w = workloads.riemann_quadrants(nx, ny, seed=1)
    with cfsb.Solver(nx, ny, precision=cfsb.FP64_EXACT) as s:
        s.set_state(w.U0)
        dts = run_counters(s, 1, 180, cfl=0.5)
        got = s.get_state()
    ref, ref_dt = ob.orc_run(ob.make_orc_config(nx, ny), w.U0, 1, 180, cfl=0.5)
    assert np.array_equal(dts, ref_dt)
    assert np.array_equal(got, ref, equal_nan=True)


def test_exact_graph_advance_equals_stepwise(cfsb, workloads):
    nx, ny = 96, 80
    w = workloads.riemann_quadrants(nx, ny, seed=7)
    with cfsb.Solver(nx, ny, precision=cfsb.FP64_EXACT) as s:
        s.set_state(w.U0)
        dts = run_counters(s, 1, 21, cfl=0.5)
        stepwise = s.get_state()
        s.set_state(w.U0)
        t, dt_last = s.advance(7, cfl=0.5)
        graph = s.get_state()
    assert np.array_equal(graph, stepwise)
    assert dt_last == dts[-1]
    assert t == pytest.approx(dts[::3].sum(), rel=1e-15)


def test_cfl_dt_is_bitwise_the_oracle(cfsb, workloads):
    nx, ny = 200, 120
    w = workloads.riemann_quadrants(nx, ny, seed=9)
    for prec in (cfsb.FP64_EXACT, cfsb.FP64):
        with cfsb.Solver(nx, ny, precision=prec) as s:
            s.set_state(w.U0)
            assert s.compute_dt(0.37) == ob.orc_cfl_dt(ob.make_orc_config(nx, ny), w.U0, 0.37)


# ------------------------------------------------------- stage, FP64 form
@pytest.mark.parametrize("rk,hll,bc", [
    (1, 0, (0, 0, 0, 0)),          # reference TVD3 + reference HLL, Neumann
    (0, 0, (1, 0, 0, 0)),          # reference TVD2, Dirichlet inflow
    (2, 1, (2, 2, 2, 2)),          # SSP-RK3, Davis HLL, periodic
    (2, 1, (2, 2, 0, 1)),          # periodic x, Neumann/Dirichlet y
])
def test_fp64_per_step_relative_linf(cfsb, workloads, rk, hll, bc):
    nx, ny = 96, 72
    w = workloads.riemann_quadrants(nx, ny, seed=3)
    cfg = ob.make_orc_config(nx, ny, rk=rk, hll=hll, bc=bc, bc_prim=[MACH3] * 4)
    S = 2 if rk == 0 else 3
    U = w.U0.copy()
    worst = 0.0
    with cfsb.Solver(nx, ny, precision=cfsb.FP64, rk=rk, hll=hll, bc=bc, bc_prim=[MACH3] * 4) as s:
        for step in range(12):
            dt = ob.orc_cfl_dt(cfg, U, 0.45)
            s.set_state(U)
            s.step(dt)
            got = s.get_state()
            ref, _ = ob.orc_run(cfg, U, 1, S, dt=dt)
            if not np.all(np.isfinite(ref)):
                break
            worst = max(worst, _rel_linf(got, ref))
            U = ref
    assert worst <= 1e-12, worst


@pytest.fixture(scope="module")
def c1_oracle_run(workloads):
    """The four-quadrant configuration at its own size (256^2, seed 1, TVD3 as
    written, reference HLL, transmissive sides, CFL 0.5): the oracle's 200
    steps (600 stages) with their dt."""
    w = workloads.riemann_quadrants(256, 256, seed=1)
    U, dts = ob.orc_run(ob.make_orc_config(256, 256), w.U0, 1, 600, cfl=0.5)
    return w, U, dts


def test_exact_form_is_bitwise_the_oracle_over_the_quadrant_configuration(cfsb, c1_oracle_run):
    """CFS_FP64_EXACT through the stage API, 600 loop iterations with the CFL
    dt at each step start: every dt and the final state equal the oracle's bit
    for bit (the oracle equals the reference's own classes, test_oracle.py)."""
    w, ref, ref_dt = c1_oracle_run
    with cfsb.Solver(256, 256, precision=cfsb.FP64_EXACT) as s:
        s.set_state(w.U0)
        dts = run_counters(s, 1, 600, cfl=0.5)
        got = s.get_state()
    assert np.array_equal(dts, ref_dt)
    assert np.array_equal(got, ref, equal_nan=True)


def test_fp64_per_step_on_the_quadrant_configuration(cfsb, c1_oracle_run):
    """CFS_FP64 at 256^2, all 200 steps: each step started from the oracle's
    state with the oracle's dt, relative L-infinity <= 1e-12 per step."""
    w, _, _ = c1_oracle_run
    cfg = ob.make_orc_config(256, 256)
    U = w.U0.copy()
    worst = 0.0
    with cfsb.Solver(256, 256, precision=cfsb.FP64) as s:
        for _ in range(200):
            dt = ob.orc_cfl_dt(cfg, U, 0.5)
            s.set_state(U)
            s.step(dt)
            got = s.get_state()
            ref, _ = ob.orc_run(cfg, U, 1, 3, dt=dt)
            assert np.all(np.isfinite(ref))
            worst = max(worst, _rel_linf(got, ref))
            U = ref
    assert worst <= 1e-12, worst


def test_fp64_full_quadrant_run_tracks_oracle(cfsb, workloads):
    """256^2 quadrant configuration, 200 steps at CFL 0.5: the FP64 form stays
    within 1e-9 relative of the oracle over the whole run (per-step error 1e-15
    amplified by the shocks)."""
    nx = ny = 256
    w = workloads.riemann_quadrants(nx, ny, seed=1)
    with cfsb.Solver(nx, ny, precision=cfsb.FP64) as s:
        s.set_state(w.U0)
        s.advance(200, cfl=0.5)
        got = s.get_state()
    ref, _ = ob.orc_run(ob.make_orc_config(nx, ny), w.U0, 1, 600, cfl=0.5)
    assert np.all(np.isfinite(got))
    assert _rel_linf(got, ref) <= 1e-9


# -------------------------------------------------- FP32-mixed form
def test_fp32_mixed_error_and_conservation(cfsb, workloads):
    """Smooth periodic advection, 256^2 to t = 0.5 (about 1,500 steps) with a
    fixed dt: density L1 error against the FP64 path <= 2e-6 (the FP32 storage
    rounding floor is a few 1e-7 here; a systematic per-step bias of 3e-8 --
    RK coefficients that do not sum to 1 in FP32 -- would already give ~6e-6),
    mass/energy drift <= 1e-6 relative."""
    n = 256
    w = workloads.smooth_advection(n)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(2, 2, 2, 2))
    cfg = ob.make_orc_config(n, n, rk=2, hll=1, bc=(2, 2, 2, 2))
    dt0 = ob.orc_cfl_dt(cfg, w.U0, 0.4)
    nsteps = int(np.ceil(0.5 / dt0))
    dt = 0.5 / nsteps
    out = {}
    for prec in (cfsb.FP64, cfsb.FP32_MIXED):
        with cfsb.Solver(n, n, precision=prec, **kw) as s:
            s.set_state(w.U0)
            m0 = s.totals()
            s.advance(nsteps, dt=dt)
            out[prec] = (s.get_state(), m0, s.totals())
    U64, U32 = out[cfsb.FP64][0], out[cfsb.FP32_MIXED][0]
    l1 = np.abs(U32[0] - U64[0]).mean()
    assert l1 <= 2e-6, l1
    _, m0, m1 = out[cfsb.FP32_MIXED]
    assert abs(m1[0] - m0[0]) / abs(m0[0]) <= 1e-6
    assert abs(m1[3] - m0[3]) / abs(m0[3]) <= 1e-6
    # and the FP64 path converges to the exact solution
    exact = workloads.smooth_advection_exact(n, 0.5)
    assert np.abs(U64[0] - exact).mean() < 1e-4
    # round-to-nearest storage (biased on this smooth, slowly moving state) is
    # the less accurate of the two FP32 roundings
    with cfsb.Solver(n, n, precision=cfsb.FP32_MIXED, rounding=cfsb.ROUND_NEAREST, **kw) as s:
        s.set_state(w.U0)
        s.advance(nsteps, dt=dt)
        l1_rn = np.abs(s.get_state()[0] - U64[0]).mean()
    assert l1 < l1_rn, (l1, l1_rn)


def test_fp32_stochastic_rounding_is_reproducible(cfsb, workloads):
    """The random bits depend on cell and step count only: two runs agree bit
    for bit, and so do one advance(6) and six advance(1) calls (the step
    counter carries across calls) and the stage-by-stage path."""
    w = workloads.smooth_advection(96)
    kw = dict(precision=cfsb.FP32_MIXED, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(2, 2, 2, 2))
    states = []
    for mode in ("one", "one", "split", "stages"):
        with cfsb.Solver(96, 96, **kw) as s:
            s.set_state(w.U0)
            if mode == "one":
                s.advance(6, dt=1e-3)
            elif mode == "split":
                for _ in range(6):
                    s.advance(1, dt=1e-3)
            else:
                for _ in range(6):
                    s.step(1e-3)
            states.append(s.get_state())
    for U in states[1:]:
        assert np.array_equal(U, states[0])


def test_fp64_slip_cylinder_per_step(cfsb, workloads):
    """Mach-3 cylinder (2 x 1 domain, 256 x 128), slip-wall immersed boundary,
    SSP-RK3 + Davis HLL, body positivity fallback (without it the scheme reaches
    negative pressure behind the body within the first step): per-step relative
    L-infinity <= 1e-12 against the oracle."""
    nx, ny = 256, 128
    w = workloads.mach3_cylinder(nx, ny)
    types, cells, donors, images, normals = cfsb.circle_setup(nx, ny, 2.0, 1.0, *w.circle, 400)
    U = w.U0.copy()  # freestream in the body too: solid cells stay inside the fluid stencils
    cfg = ob.make_orc_config(nx, ny, lx=2.0, ly=1.0, rk=2, hll=1, bc=w.bc, bc_prim=w.bc_prim, positivity=2)
    ib = ob.OrcIBList(cells, donors, images, normals, mode=1, types=types)
    worst = 0.0
    with cfsb.Solver(nx, ny, 2.0, 1.0, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=w.bc,
                     bc_prim=w.bc_prim, positivity=cfsb.POSITIVITY_BODY) as s:
        s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP)
        for _ in range(10):
            dt = ob.orc_cfl_dt(cfg, U, 0.5, types)
            s.set_state(U)
            s.step(dt)
            got = s.get_state()
            ref, _ = ob.orc_run(cfg, U, 1, 3, dt=dt, types=types, ib=ib)
            assert np.all(np.isfinite(ref))
            worst = max(worst, _rel_linf(got, ref))
            U = ref
    assert worst <= 1e-12, worst


@pytest.mark.parametrize("prec", [0, 1])
def test_body_positivity_keeps_mach3_cylinder_physical(cfsb, workloads, prec):
    """300 steps of the Mach-3 cylinder (256 x 128, CFL 0.5) with the body
    positivity fallback stay finite with positive density and pressure."""
    w = workloads.mach3_cylinder(256, 128)
    with cfsb.Solver(256, 128, 2.0, 1.0, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=w.bc,
                     bc_prim=w.bc_prim, positivity=cfsb.POSITIVITY_BODY) as s:
        s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP)
        types, *_ = cfsb.circle_setup(256, 128, 2.0, 1.0, *w.circle, 400)
        s.set_state(w.U0)
        t, _ = s.advance(300, cfl=0.5)
        U = s.get_state()
    f = types == 0
    p = 0.4 * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0])
    assert np.all(np.isfinite(U[:, f])) and t > 0
    assert U[0][f].min() > 0 and p[f].min() > 0


def _rarefaction(workloads, nx=64, ny=48, speed=4.0):
    """Two halves moving apart at +-speed (rho 1, p 0.4): a near-vacuum forms
    between them, where the reference's scheme reaches negative pressure."""
    X, _ = workloads.cell_centres(nx, ny, 1.0, 1.0)
    return workloads.conserved(np.ones((nx, ny)), np.where(X < 0.5, -speed, speed), 0.0, 0.4)


def test_fp64_floor_per_step(cfsb, workloads):
    """CFS_POSITIVITY_FLOOR against the oracle's floors, per step from the
    oracle's state with its dt, through the near-vacuum where the floors act.
    Whether a cell sits just above or below a floor can differ by rounding, so:
    relative L-infinity <= 1e-12 on cells more than 4 cells (3 stages of a
    3-cell stencil) from any near-floor cell, <= 1e-5 of the state's magnitude
    everywhere, and the result finite with positive density and pressure."""
    U = _rarefaction(workloads)
    cfg = ob.make_orc_config(64, 48, rk=2, hll=1, positivity=3)
    worst_far, worst_all, floored = 0.0, 0.0, False
    with cfsb.Solver(64, 48, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     positivity=cfsb.POSITIVITY_FLOOR) as s:
        for _ in range(20):
            dt = ob.orc_cfl_dt(cfg, U, 0.5)
            s.set_state(U)
            s.step(dt)
            got = s.get_state()
            ref, _ = ob.orc_run(cfg, U, 1, 3, dt=dt)
            assert np.all(np.isfinite(ref)) and np.all(np.isfinite(got))
            near = np.zeros(U.shape[1:], dtype=bool)
            for X in (U, ref, got):
                pX = 0.4 * (X[3] - 0.5 * (X[1] ** 2 + X[2] ** 2) / X[0])
                near |= (X[0] < 1e-4) | (pX < 1e-4)
            floored = floored or bool(near.any())
            grow = near.copy()
            for _k in range(4):
                g2 = grow.copy()
                g2[1:] |= grow[:-1]
                g2[:-1] |= grow[1:]
                g2[:, 1:] |= grow[:, :-1]
                g2[:, :-1] |= grow[:, 1:]
                grow = g2
            scale = np.abs(ref).max()
            d = np.abs(got - ref) / scale
            worst_all = max(worst_all, float(d.max()))
            if (~grow).any():
                worst_far = max(worst_far, float(d[:, ~grow].max()))
            pg = 0.4 * (got[3] - 0.5 * (got[1] ** 2 + got[2] ** 2) / got[0])
            assert got[0].min() > 0 and pg.min() > 0
            U = ref
    assert floored, "the floors never acted"
    assert worst_far <= 1e-12, worst_far
    assert worst_all <= 1e-5, worst_all


def test_fp32_floor_keeps_rarefaction_finite(cfsb, workloads):
    U = _rarefaction(workloads)
    with cfsb.Solver(64, 48, precision=cfsb.FP32_MIXED, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     positivity=cfsb.POSITIVITY_FLOOR) as s:
        s.set_state(U)
        s.advance(60, cfl=0.5)
        V = s.get_state()
    assert np.all(np.isfinite(V)) and V[0].min() > 0
