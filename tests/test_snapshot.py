"""Snapshot writer (Output::WriteToHDF5 layout, Output.cpp:8-90): dataset
names, x-major (Nx, Ny) order and contents, checked against the reference's own
cell data after a short run (the values its writer reads, Output.cpp:60-74)."""
import importlib
import json

import numpy as np
import pytest

import oracle_bind as ob

snap = importlib.import_module("2d_compressible_flow_solver_b200.snapshot")


def test_raw_snapshot_layout_and_round_trip(tmp_path, workloads):
    w = workloads.riemann_quadrants(24, 16, seed=2)
    U, rhs, _ = ob.ref_run(24, 16, w.U0, 3, integrator=3, dt=1e-3)
    p = snap.write_snapshot(tmp_path / "s", U, rhs, time=3e-3, fmt="raw")
    index = json.loads((p / "index.json").read_text())
    assert index["datasets"] == list(snap.DATASETS) and index["shape"] == [24, 16]
    assert (p / "Rho.f64").stat().st_size == 24 * 16 * 8
    raw = np.fromfile(p / "Mu.f64", dtype="<f8")
    assert raw[5 * 16 + 7] == U[1][5, 7]  # x-major: (i, j) at i * ny + j
    d = snap.read_snapshot(p)
    assert np.array_equal(d["Rho"], U[0]) and np.array_equal(d["Mv"], U[2]) and np.array_equal(d["Energy"], U[3])
    assert np.array_equal(d["FluxRho"], rhs[0]) and np.array_equal(d["FluxEnergy"], rhs[3])
    pr = 0.4 * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0])
    assert np.allclose(d["Pressure"], pr, rtol=1e-15, atol=0)
    assert not d["Udir"].any() and not d["Vdir"].any() and not d["Tdir"].any()


def test_pressure_of_unfilled_solid_cells_is_zero():
    U = np.zeros((4, 3, 3))
    U[:, 1, 1] = [1.0, 0.5, 0.0, 2.5]
    d = snap.snapshot_arrays(U)
    assert d["Pressure"][0, 0] == 0.0 and d["Pressure"][1, 1] == pytest.approx(0.4 * (2.5 - 0.125))


def test_rejects_bad_shapes():
    with pytest.raises(ValueError):
        snap.snapshot_arrays(np.zeros((3, 4, 4)))
    with pytest.raises(ValueError):
        snap.snapshot_arrays(np.zeros((4, 4, 4)), np.zeros((4, 3, 4)))


@pytest.mark.gpu
def test_solver_snapshot_matches_reference_writer_inputs(cfsb, workloads, tmp_path):
    """An exact-form engine run written through write_solver_snapshot holds what
    the reference's writer would read from its cells after the same stages."""
    w = workloads.riemann_quadrants(64, 40, seed=6)
    U_ref, rhs_ref, _ = ob.ref_run(64, 40, w.U0, 6, integrator=3, dt=1e-3)
    with cfsb.Solver(64, 40, precision=cfsb.FP64_EXACT, keep_rhs=True) as s:
        s.set_state(w.U0)
        for k in range(1, 7):
            s.stage(k, 1e-3)
        p = snap.write_solver_snapshot(s, tmp_path / "g", fmt="raw")
    d = snap.read_snapshot(p)
    assert np.array_equal(d["Rho"], U_ref[0]) and np.array_equal(d["Mu"], U_ref[1])
    assert np.array_equal(d["FluxMu"], rhs_ref[1]) and np.array_equal(d["FluxEnergy"], rhs_ref[3])
