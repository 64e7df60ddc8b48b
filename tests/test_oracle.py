"""The C oracle (oracle/cfs_oracle.c) against the reference solver's own outputs:
the committed golden fixtures (tests/golden, produced by the reference's classes)
and, where the reference library is built here, live runs on fresh seeds.
Bit-exact equality is required: the oracle restates the reference's operation
order and is built without FMA contraction."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

GOLD = Path(__file__).resolve().parent / "golden"
MACH3 = (1.4, 3.0, 0.0, 1.0)
has_ref = ob.REF_STRICT.exists() or ob.REFERENCE_TREE is not None


def _load(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def _rk(integrator):
    return ob.RK_TVD2 if int(integrator) == 2 else ob.RK_TVD3_REFERENCE


@pytest.mark.parametrize("name", ["quadrants_tvd3_48x40_cfl", "quadrants_tvd2_32x32_cfl",
                                  "quadrants_dirichlet_tvd3_40x32"])
def test_oracle_reproduces_reference_fixture(name):
    g = _load(name)
    nx, ny, nst = int(g["cfg_nx"]), int(g["cfg_ny"]), int(g["cfg_nstages"])
    bc = tuple(int(b) for b in g.get("cfg_bc", np.zeros(4)))
    bc_prim = g["cfg_bc_prim"] if "cfg_bc_prim" in g else None
    cfg = ob.make_orc_config(nx, ny, rk=_rk(g["cfg_integrator"]), bc=bc, bc_prim=bc_prim)
    cfl = float(g.get("cfg_cfl", 0.0))
    dt = float(g.get("cfg_dt", 1e-3))
    U, dts = ob.orc_run(cfg, g["U0"], 1, nst, dt=dt, cfl=cfl)
    assert np.array_equal(dts, g["dt"])
    assert np.array_equal(U, g["U"]), f"max diff {np.abs(U - g['U']).max()}"


def test_oracle_reproduces_reference_circle_fixture():
    g = _load("circle_tvd3_64x64")
    lst = _load("circle_64x64_lists")
    nx, ny = 64, 64
    cfg = ob.make_orc_config(nx, ny, bc=(1, 0, 0, 0), bc_prim=[MACH3] * 4)
    ib = ob.OrcIBList(lst["cells"], lst["donors"], lst["images"])
    U, _ = ob.orc_run(cfg, g["U0"], 1, int(g["cfg_nstages"]), dt=float(g["cfg_dt"]), types=lst["types"], ib=ib)
    assert np.array_equal(U, g["U"], equal_nan=True)


def test_weno_face_matches_reference_fixture():
    g = _load("faces_weno_hll")
    lib = ob.orc_lib()
    for f in range(g["stencils"].shape[0]):
        s = g["stencils"][f]
        for q in range(4):
            left = lib.orc_weno5(np.ascontiguousarray(s[0:5, q]).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1e-2)
            right = lib.orc_weno5(np.ascontiguousarray(s[5:0:-1, q]).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  1e-2)
            assert left == g["left"][f, q] and right == g["right"][f, q]


def test_hll_matches_reference_fixture():
    g = _load("faces_weno_hll")
    cfg = ob.make_orc_config(8, 8)
    lib = ob.orc_lib()
    for d in range(2):
        for f in range(g["L"].shape[0]):
            out = np.empty(4)
            lib.orc_hll(ctypes.byref(cfg), ob.P(np.ascontiguousarray(g["L"][f])), ob.P(np.ascontiguousarray(g["R"][f])),
                        d, ob.P(out))
            assert np.array_equal(out, g["F"][d, f])


def test_viscous_reference_matches_fixture():
    g = _load("viscous_reference_24x20")
    nx, ny = 24, 20
    cfg = ob.make_orc_config(nx, ny, mu=1e-3, mach=1.0)
    grad = np.zeros((6, nx, ny))
    fvx = np.zeros((4, nx + 1, ny))
    fvy = np.zeros((4, nx, ny + 1))
    ob.orc_lib().orc_viscous_reference(ctypes.byref(cfg), ob.P(np.ascontiguousarray(g["U0"])), ob.P(grad), ob.P(fvx),
                                       ob.P(fvy))
    assert np.array_equal(grad, g["grad"])
    assert np.array_equal(fvx, g["fvx"])
    assert np.array_equal(fvy, g["fvy"])


@pytest.mark.skipif(not has_ref, reason="reference library not built here")
@pytest.mark.parametrize("seed,integrator,bc", [(21, 3, (0, 0, 0, 0)), (22, 2, (0, 0, 0, 0)),
                                                (23, 3, (1, 0, 1, 0)), (24, 3, (0, 1, 0, 1))])
def test_oracle_matches_live_reference(workloads, seed, integrator, bc):
    nx, ny = 36, 28
    w = workloads.riemann_quadrants(nx, ny, seed=seed)
    kw = dict(integrator=integrator, cfl=0.45, bc=bc, bc_prim=[MACH3] * 4)
    ref_U, ref_rhs, ref_dt = ob.ref_run(nx, ny, w.U0, 9, **kw)
    cfg = ob.make_orc_config(nx, ny, rk=_rk(integrator), bc=bc, bc_prim=[MACH3] * 4)
    U, dts = ob.orc_run(cfg, w.U0, 1, 9, cfl=0.45)
    assert np.array_equal(dts, ref_dt)
    assert np.array_equal(U, ref_U, equal_nan=True)


@pytest.mark.skipif(not has_ref, reason="reference library not built here")
def test_oracle_rhs_matches_reference_m_flux(workloads):
    """The RHS the reference keeps in Cell::m_flux (written as FluxRho etc.)."""
    nx, ny = 30, 26
    w = workloads.riemann_quadrants(nx, ny, seed=4)
    _, ref_rhs, _ = ob.ref_run(nx, ny, w.U0, 1, integrator=3, dt=1e-3)
    cfg = ob.make_orc_config(nx, ny)
    U = w.U0.copy()
    U0 = np.zeros_like(U)
    U1 = np.zeros_like(U)
    R = np.zeros_like(U)
    ob.orc_stage(cfg, U, U0, U1, 0, 1e-3, rhs=R)
    assert np.array_equal(R, ref_rhs)


def test_free_stream_is_preserved():
    nx, ny = 24, 24
    U0 = np.empty((4, nx, ny))
    U0[:] = np.array(ob.dirichlet_conserved(MACH3))[:, None, None]
    cfg = ob.make_orc_config(nx, ny, bc=(1, 0, 0, 0), bc_prim=[MACH3] * 4)
    U, _ = ob.orc_run(cfg, U0, 1, 12, dt=1e-3)
    assert np.allclose(U, U0, rtol=1e-14, atol=0)


def test_weno_reproduces_linear_data():
    lib = ob.orc_lib()
    for a, b in [(1.0, 0.5), (-2.0, 3.0), (0.3, -0.01)]:
        v = np.array([a + b * k for k in range(5)])
        got = lib.orc_weno5(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1e-2)
        assert abs(got - (a + b * 2.5)) <= 1e-14 * max(1.0, abs(a + b * 2.5))


def test_hll_consistency_equal_states():
    cfg = ob.make_orc_config(8, 8)
    lib = ob.orc_lib()
    rng = np.random.default_rng(3)
    for _ in range(50):
        rho, u, v, p = rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2)
        U = np.array(ob.dirichlet_conserved((rho, u, v, p)))
        for d in range(2):
            out = np.empty(4)
            lib.orc_hll(ctypes.byref(cfg), ob.P(U), ob.P(U), d, ob.P(out))
            q = U[1 + d]
            un = q / rho
            exact = np.array([q, U[1] * un + (p if d == 0 else 0), U[2] * un + (p if d == 1 else 0), (U[3] + p) * un])
            assert np.allclose(out, exact, rtol=1e-13, atol=1e-15)


def test_positivity_fallback_on_mach3_cylinder(cfsb):
    """The reference scheme (no fallback) reaches NaN on the Mach-3 cylinder in
    its first step; the body fallback keeps 40 steps finite."""
    import importlib
    wl = importlib.import_module("2d_compressible_flow_solver_b200.workloads")
    nx, ny = 128, 64
    w = wl.mach3_cylinder(nx, ny)
    types, cells, donors, images, normals = cfsb.circle_setup(nx, ny, 2.0, 1.0, *w.circle, 400)
    ib = ob.OrcIBList(cells, donors, images, normals, mode=1, types=types)
    f = types == 0
    finite = {}
    for pos, nsteps in ((0, 1), (2, 40)):
        cfg = ob.make_orc_config(nx, ny, lx=2.0, ly=1.0, rk=2, hll=1, bc=w.bc, bc_prim=w.bc_prim, positivity=pos)
        U = w.U0.copy()
        for _ in range(nsteps):
            dt = ob.orc_cfl_dt(cfg, U, 0.5, types)
            U, _ = ob.orc_run(cfg, U, 1, 3, dt=dt, types=types, ib=ib)
        finite[pos] = bool(np.all(np.isfinite(U[:, f])))
    assert finite == {0: False, 2: True}


def test_floors_carry_a_near_vacuum(workloads):
    """Two halves moving apart at +-4 (rho 1, p 0.4): without floors the oracle
    reaches NaN within 10 steps; with them (ORC_POS_FLOOR) 40 steps stay finite
    and the pressure floor is reached."""
    X, _ = workloads.cell_centres(64, 48, 1.0, 1.0)
    U0 = workloads.conserved(np.ones((64, 48)), np.where(X < 0.5, -4.0, 4.0), 0.0, 0.4)
    out = {}
    for pos in (2, 3):
        cfg = ob.make_orc_config(64, 48, rk=2, hll=1, positivity=pos)
        U = U0.copy()
        pmin = np.inf
        for _ in range(40):
            U, _ = ob.orc_run(cfg, U, 1, 3, dt=ob.orc_cfl_dt(cfg, U, 0.5))
            with np.errstate(invalid="ignore"):
                pmin = min(pmin, float(np.nanmin(0.4 * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0]))))
            if not np.all(np.isfinite(U)):
                break
        out[pos] = (bool(np.all(np.isfinite(U))), pmin)
    assert out[2][0] is False
    assert out[3][0] is True and out[3][1] <= 1.0000001e-6
