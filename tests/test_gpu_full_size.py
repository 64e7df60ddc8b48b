"""The configured workloads at their full sizes, checked through properties
that hold at any size (the oracle finishes only small grids in seconds):

* smooth periodic advection at 4096 x 4096 (the bandwidth run): the state
  depends on x + y only and u = v, so every cell must equal its diagonal
  neighbour and the x- and y-momentum must agree; the FP64 form against the
  exact translated solution; conservation of every total on periodic sides;
  FP32-mixed against FP64 on one time-step sequence, and its mass drift;
* the Mach-3 cylinder at 2048 x 1024: the body is centred on y = 1/2 and the
  inflow has v = 0, so the flow is mirror-symmetric about that line (the
  immersed-boundary set-up is, exactly: tests/test_ib_setup.py); positive
  density and pressure in every fluid cell; FP32-mixed against FP64;
* the Navier-Stokes shear layer at 1024 x 1024: mass, both momenta and energy
  conserved on periodic sides with the viscous fluxes on; FP32-mixed against
  FP64;
* the uneven 512-case batch: every case finite with positive density, and
  sampled cases equal to the same case advanced alone.

Each run is a few tens of steps, so the time the suite takes stays small; the
long runs to the configured end times are the benchmark's report.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def _fp64_dts(cfsb, w, steps, cfl, **kw):
    """FP64 run with CFL steps: (state, totals before, totals after, dt sequence)."""
    with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=cfsb.FP64, bc=w.bc, bc_prim=w.bc_prim, **kw) as s:
        if w.circle is not None:
            s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP)
        s.set_state(w.U0)
        m0 = s.totals()
        dts = np.array([s.advance(1, cfl=cfl)[1] for _ in range(steps)])
        return s.get_state(), m0, s.totals(), dts


def _replay(cfsb, w, prec, dts, **kw):
    """The same workload in another form, replaying a dt sequence."""
    with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, bc=w.bc, bc_prim=w.bc_prim, **kw) as s:
        if w.circle is not None:
            s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP)
        s.set_state(w.U0)
        m0 = s.totals()
        for dt in dts:
            s.advance(1, dt=float(dt))
        return s.get_state(), m0, s.totals()


def _rel_change(m0, m1, scale=None):
    scale = np.abs(m0) if scale is None else scale
    return np.abs(m1 - m0) / scale


def smooth_advection_4096(cfsb, wl, steps=16):
    w = wl.smooth_advection(4096)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS)
    U64, a0, a1, dts = _fp64_dts(cfsb, w, steps, w.cfl, **kw)
    U32, b0, b1 = _replay(cfsb, w, cfsb.FP32_MIXED, dts, **kw)
    t = float(dts.sum())
    diag = np.roll(np.roll(U64, -1, axis=1), 1, axis=2)        # U[:, i+1, j-1]
    exact = wl.smooth_advection_exact(4096, t)
    scale = np.array([abs(a0[0]), abs(a0[0]), abs(a0[0]), abs(a0[3])])   # momenta start equal to the mass
    return {
        "t": t,
        "diagonal_max": float(np.abs(diag - U64).max()),
        "mx_vs_my_max": float(np.abs(U64[1] - U64[2]).max()),
        "fp64_vs_exact_L1": float(np.abs(U64[0] - exact).mean()),
        "fp64_totals_change": _rel_change(a0, a1, scale).tolist(),
        "fp32_rho_L1": float(np.abs(U32[0] - U64[0]).mean()),
        "fp32_rho_Linf": float(np.abs(U32[0] - U64[0]).max()),
        "fp32_E_L1": float(np.abs(U32[3] - U64[3]).mean()),
        "fp32_mass_drift": float(abs(b1[0] - b0[0]) / abs(b0[0])),
        "finite": bool(np.isfinite(U64).all() and np.isfinite(U32).all()),
    }


def _pressure(U):
    return (GAMMA - 1.0) * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0])


def mach3_cylinder_2048(cfsb, wl, steps=40):
    w = wl.mach3_cylinder(2048, 1024)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, positivity=cfsb.POSITIVITY_FLOOR)
    U64, _, _, dts = _fp64_dts(cfsb, w, steps, w.cfl, **kw)
    U32, _, _ = _replay(cfsb, w, cfsb.FP32_MIXED, dts, **kw)
    types = cfsb.circle_setup(w.nx, w.ny, w.lx, w.ly, *w.circle, 400)[0]
    fluid = types == 0
    mirror = U64[:, :, ::-1].copy()
    mirror[2] = -mirror[2]
    sym = np.abs(U64 - mirror)[:, fluid]
    moved = np.abs(U64 - w.U0)[0][fluid]
    return {
        "t": float(dts.sum()),
        "finite": bool(np.isfinite(U64).all() and np.isfinite(U32).all()),
        "fp64_min_rho": float(U64[0][fluid].min()), "fp64_min_p": float(_pressure(U64)[fluid].min()),
        "fp32_min_rho": float(U32[0][fluid].min()), "fp32_min_p": float(_pressure(U32)[fluid].min()),
        "mirror_max": [float(x) for x in sym.max(axis=1)],
        "flow_moved_max": float(moved.max()),
        "fp32_rho_L1": float(np.abs(U32[0] - U64[0])[fluid].mean()),
        "fp32_rho_Linf": float(np.abs(U32[0] - U64[0])[fluid].max()),
    }


def shear_layer_1024(cfsb, wl, steps=20):
    w = wl.shear_layer(1024)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, viscous=cfsb.VISCOUS_NS, mu=w.meta["mu"], prandtl=0.72,
              mach=1.0)
    U64, a0, a1, dts = _fp64_dts(cfsb, w, steps, w.cfl, **kw)
    U32, b0, b1 = _replay(cfsb, w, cfsb.FP32_MIXED, dts, **kw)
    scale = np.abs(w.U0).reshape(4, -1).sum(axis=1) * (1.0 / (w.nx * w.ny))   # totals are cell means
    return {
        "t": float(dts.sum()),
        "finite": bool(np.isfinite(U64).all() and np.isfinite(U32).all()),
        "fp64_totals_change": _rel_change(a0, a1, scale).tolist(),
        "fp32_totals_change": _rel_change(b0, b1, scale).tolist(),
        "totals_scale": scale.tolist(), "totals0": a0.tolist(),
        "fp32_rho_L1": float(np.abs(U32[0] - U64[0]).mean()),
        "fp32_rho_Linf": float(np.abs(U32[0] - U64[0]).max()),
    }


def batch_512(cfsb, wl, steps=3, sample=(0, 1, 2, 3)):
    """The uneven batch in FP32-mixed: per-case CFL steps; the cases named by
    `sample` (positions in size order, smallest and largest first) advanced
    alone on each case's own dt sequence replayed."""
    cases, states = wl.batch_cases(512, seed=1)
    dts = []
    with cfsb.Batch(cases, precision=cfsb.FP32_MIXED, positivity=cfsb.POSITIVITY_FLOOR) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        for _ in range(steps):
            b.advance(1, cfl=0.5)
            dts.append(b.dt_last())
        got = [b.get_state(k) for k in range(len(cases))]
    dts = np.array(dts)
    finite = all(np.isfinite(U).all() for U in got)
    min_rho = min(float(U[0].min()) for U in got)
    by_size = sorted(range(len(cases)), key=lambda k: cases[k]["nx"] * cases[k]["ny"])
    picks = [by_size[0], by_size[-1], by_size[len(by_size) // 3], by_size[(2 * len(by_size)) // 3]]
    picks = [picks[i] for i in sample]
    diffs = {}
    for k in picks:
        c = cases[k]
        with cfsb.Solver(c["nx"], c["ny"], c["lx"], c["ly"], precision=cfsb.FP32_MIXED, rk=cfsb.RK_SSP3,
                         hll=cfsb.HLL_DAVIS, bc=c["bc"], bc_prim=c.get("bc_prim"),
                         positivity=cfsb.POSITIVITY_FLOOR) as s:
            if "circle" in c:
                s.build_circle(*c["circle"], 400, cfsb.IB_BILINEAR_SLIP)
            s.set_state(states[k])
            for dt in dts[:, k]:
                s.advance(1, dt=float(dt))
            ref = s.get_state()
        diffs[f"{k}:{c['nx']}x{c['ny']}"] = float(np.abs(got[k] - ref).max() / np.abs(ref).max())
    return {"finite": finite, "min_rho": min_rho, "cells": int(sum(c["nx"] * c["ny"] for c in cases)),
            "sample_rel_max_diff": diffs, "dt_min": float(dts.min()), "dt_max": float(dts.max())}


# Bounds: each sits one to two orders of magnitude above what these runs
# measure on a B200 (in brackets), so any indexing, halo or boundary fault,
# which moves values by O(1e-3) or more, fails them.

def test_smooth_advection_4096_properties(cfsb, workloads):
    r = smooth_advection_4096(cfsb, workloads)
    assert r["finite"]
    # position-independent to a few ulps, not to the bit (most departures sit
    # within three cells of the periodic edges) [5.3e-15, 1.8e-15]
    assert r["diagonal_max"] <= 1e-13, r
    assert r["mx_vs_my_max"] <= 1e-13, r
    assert r["fp64_vs_exact_L1"] <= 1e-13, r                  # [1.0e-15 at t = 3.4e-4]
    assert max(r["fp64_totals_change"]) <= 1e-14, r           # [1.3e-16]
    assert r["fp32_rho_L1"] <= 5e-7 and r["fp32_rho_Linf"] <= 5e-6, r   # [4.9e-8, 5.1e-7]
    assert r["fp32_mass_drift"] <= 1e-10, r                   # [1.2e-12]


def test_mach3_cylinder_2048x1024_properties(cfsb, workloads):
    r = mach3_cylinder_2048(cfsb, workloads)
    assert r["finite"]
    assert r["flow_moved_max"] > 1.0, r                       # the bow shock has formed [4.4]
    assert min(r["fp64_min_rho"], r["fp64_min_p"], r["fp32_min_rho"], r["fp32_min_p"]) > 0.0, r
    assert max(r["mirror_max"]) <= 1e-8, r                    # [2.7e-10, energy]
    assert r["fp32_rho_L1"] <= 1e-7 and r["fp32_rho_Linf"] <= 1e-4, r   # [1.1e-8, 3.3e-6]


def test_shear_layer_1024_navier_stokes_properties(cfsb, workloads):
    r = shear_layer_1024(cfsb, workloads)
    assert r["finite"]
    assert max(r["fp64_totals_change"]) <= 1e-13, r           # [6.6e-16]
    assert max(r["fp32_totals_change"]) <= 1e-8, r           # [1.8e-10, the momenta]
    assert r["fp32_rho_L1"] <= 2e-7 and r["fp32_rho_Linf"] <= 2e-6, r   # [1.9e-8, 1.6e-7]


def test_batch_512_cases_properties(cfsb, workloads):
    r = batch_512(cfsb, workloads)
    assert r["finite"] and r["min_rho"] > 0.0, r
    assert r["cells"] == 90952704
    assert max(r["sample_rel_max_diff"].values()) <= 1e-6, r  # [5.0e-8]
