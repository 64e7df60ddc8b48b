"""Generates the golden fixtures in this folder from the reference solver's own
classes (oracle/_ref/libref_strict.so, built by oracle/Makefile from the
reference tree with -O2 -ffp-contract=off against the repo's Eigen/MPI shims).

The reference ships no tests or golden data, so these fixtures ARE its outputs,
captured here once and committed; the GPU box never needs the reference tree.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle_bind as ob  # noqa: E402

wl = importlib.import_module("2d_compressible_flow_solver_b200.workloads")

MACH3 = (1.4, 3.0, 0.0, 1.0)


def run_case(name, nx, ny, U0, nstages, **kw):
    out, rhs, dts = ob.ref_run(nx, ny, U0, nstages, **kw)
    cfg = dict(nx=nx, ny=ny, nstages=nstages, **{k: v for k, v in kw.items() if k != "bc_prim"})
    if "bc_prim" in kw:
        cfg["bc_prim"] = np.asarray(kw["bc_prim"], dtype=np.float64)
    np.savez_compressed(HERE / f"{name}.npz", U0=U0, U=out, rhs=rhs, dt=dts,
                        **{f"cfg_{k}": np.asarray(v) for k, v in cfg.items() if k != "circle"},
                        **({"cfg_circle": np.asarray(kw["circle"])} if "circle" in kw else {}))
    print(name, "nan:", int(np.isnan(out).sum()))


def main():
    # Four-quadrant Riemann states (the seeded first configuration), Neumann sides.
    w = wl.riemann_quadrants(48, 40, seed=3)
    run_case("quadrants_tvd3_48x40_cfl", 48, 40, w.U0, 30, integrator=3, cfl=0.5)
    w = wl.riemann_quadrants(32, 32, seed=1)
    run_case("quadrants_tvd2_32x32_cfl", 32, 32, w.U0, 20, integrator=2, cfl=0.5)
    # Dirichlet Mach-3 inflow on the left, fixed dt.
    w = wl.riemann_quadrants(40, 32, seed=2)
    run_case("quadrants_dirichlet_tvd3_40x32", 40, 32, w.U0, 12, integrator=3, dt=2e-3,
             bc=(1, 0, 0, 0), bc_prim=[MACH3] * 4)
    # Immersed circle (reference LDLT fill), a few stages before the reference's
    # non-interpolating fill drives the state to NaN.
    nx = ny = 64
    types, cells, donors, images, nd = ob.ref_ib_info(nx, ny, 1.0, 1.0, (0.2, 0.45, 0.55))
    w = wl.riemann_quadrants(nx, ny, seed=5)
    U0 = w.U0.copy()
    U0[:, types != 0] = 0.0  # the reference fills the initial condition on fluid cells only
    run_case("circle_tvd3_64x64", nx, ny, U0, 2, integrator=3, dt=1e-3, bc=(1, 0, 0, 0),
             bc_prim=[MACH3] * 4, circle=(0.2, 0.45, 0.55))
    np.savez_compressed(HERE / "circle_64x64_lists.npz", types=types, cells=cells, donors=donors, images=images,
                        n_donors=nd, circle=np.array([0.2, 0.45, 0.55]), grid=np.array([nx, ny, 1.0, 1.0]))
    # Full-size immersed-boundary lists of the Mach-3 cylinder configuration.
    nx, ny = 2048, 1024
    types, cells, donors, images, nd = ob.ref_ib_info(nx, ny, 2.0, 1.0, (0.05, 0.4, 0.5))
    np.savez_compressed(HERE / "cylinder_2048x1024_lists.npz", solid=np.flatnonzero(types == 1).astype(np.int32),
                        cells=cells, donors=donors, images=images, n_donors=nd,
                        circle=np.array([0.05, 0.4, 0.5]), grid=np.array([nx, ny, 2.0, 1.0]))
    print("cylinder IG cells:", cells.size)

    # Unit-level: WENO faces and HLL faces through the reference's plugin calls.
    rng = np.random.default_rng(11)
    n = 256
    st = np.empty((n, 6, 4))
    st[:, :, 0] = rng.uniform(0.2, 2.0, (n, 6))
    st[:, :, 1] = st[:, :, 0] * rng.uniform(-1.5, 1.5, (n, 6))
    st[:, :, 2] = st[:, :, 0] * rng.uniform(-1.5, 1.5, (n, 6))
    p = rng.uniform(0.1, 2.0, (n, 6))
    st[:, :, 3] = p / 0.4 + 0.5 * (st[:, :, 1] ** 2 + st[:, :, 2] ** 2) / st[:, :, 0]
    st[:32] = st[:32, :1, :]  # constant stencils
    left = np.empty((n, 5))
    right = np.empty((n, 5))
    lib = ob.ref_lib()
    for f in range(n):
        s = np.ascontiguousarray(st[f])
        lo = np.empty(5)
        ro = np.empty(5)
        lib.ref_weno_face(ob.P(s), ob.P(lo), ob.P(ro))
        left[f], right[f] = lo, ro
    L = st[:, 2, :].copy()
    R = st[:, 3, :].copy()
    F = np.empty((2, n, 4))
    for d in range(2):
        for f in range(n):
            out = np.empty(4)
            lib.ref_hll(ob.P(np.ascontiguousarray(L[f])), ob.P(np.ascontiguousarray(R[f])), d, ob.P(out))
            F[d, f] = out
    np.savez_compressed(HERE / "faces_weno_hll.npz", stencils=st, left=left, right=right, L=L, R=R, F=F)

    # The reference's (unwired) viscous routines on a smooth state, Neumann sides.
    nx, ny = 24, 20
    X, Y = wl.cell_centres(nx, ny, 1.0, 1.0)
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    u = 0.3 * np.sin(2 * np.pi * Y)
    v = 0.2 * np.cos(2 * np.pi * X)
    pr = 1.0 + 0.1 * np.cos(2 * np.pi * (X + Y))
    U0 = wl.conserved(rho, u, v, pr)
    c = ob.make_ref_config(nx, ny)
    grad = np.zeros((6, nx, ny))
    fvx = np.zeros((4, nx + 1, ny))
    fvy = np.zeros((4, nx, ny + 1))
    lib.ref_viscous(ctypes.byref(c), ob.P(U0), ob.P(grad), ob.P(fvx), ob.P(fvy))
    np.savez_compressed(HERE / "viscous_reference_24x20.npz", U0=U0, grad=grad, fvx=fvx, fvy=fvy)


if __name__ == "__main__":
    main()
