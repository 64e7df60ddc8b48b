"""Snapshot writer with the reference's output layout
(Output::WriteToHDF5, source/io/Output.cpp:8-90).

The reference writes twelve FP64 datasets of shape (Nx, Ny), x-major
(index i * Ny + j, Output.cpp:60): Mu, Mv (momenta), Rho, Energy (total
energy), Pressure, FluxMu, FluxMv, FluxRho, FluxEnergy (the RHS each cell holds
from its last stage, Cell.cpp:135-137), and Udir = du/dx, Vdir = dv/dy,
Tdir = dT/dx from the cell gradients.  The reference's loop never computes
those gradients (Run.cpp:176-180 has the call commented out), so its files
hold zeros there, and so do these.

HDF5 is written when h5py is importable (same dataset names); otherwise the
same datasets are written raw: ``<dir>/<Name>.f64`` (little-endian float64,
Nx * Ny values in the order above) plus ``<dir>/index.json`` describing them.

A snapshot may also carry the run's counters (no reference counterpart: the
reference writes snapshots and never reads them back, Output.cpp:20): time,
last dt, completed steps, the CFL maximum the next step would use and the
FP32-mixed storage offsets -- what a new engine context needs to continue the
run bit for bit (``resume_solver``).  Raw: the ``run`` entry of index.json;
HDF5: attributes of the file.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

DATASETS = ("Mu", "Mv", "Rho", "Energy", "Pressure", "FluxMu", "FluxMv", "FluxRho", "FluxEnergy",
            "Udir", "Vdir", "Tdir")


def snapshot_arrays(U: np.ndarray, rhs: np.ndarray | None = None, gamma: float = 1.4) -> dict[str, np.ndarray]:
    """The twelve datasets from a conserved state U[4][nx][ny] and (optional)
    RHS[4][nx][ny].  Pressure follows EulerPhase::computePressurefromOther
    (EulerPhase.cpp:130-133); cells with rho == 0 (solid cells the reference
    never fills, Run.cpp:98-104) get 0 as their never-computed pressure."""
    U = np.asarray(U, dtype=np.float64)
    if U.ndim != 3 or U.shape[0] != 4:
        raise ValueError("U must have shape (4, nx, ny)")
    rho, mx, my, E = U
    with np.errstate(divide="ignore", invalid="ignore"):
        p = np.where(rho != 0.0, (gamma - 1.0) * (E - 0.5 * (mx * mx + my * my) / rho), 0.0)
    R = np.zeros_like(U) if rhs is None else np.asarray(rhs, dtype=np.float64)
    if R.shape != U.shape:
        raise ValueError("rhs must have the state's shape")
    z = np.zeros_like(rho)
    return {"Mu": mx, "Mv": my, "Rho": rho, "Energy": E, "Pressure": p, "FluxMu": R[1], "FluxMv": R[2],
            "FluxRho": R[0], "FluxEnergy": R[3], "Udir": z, "Vdir": z, "Tdir": z}


def write_snapshot(path, U: np.ndarray, rhs: np.ndarray | None = None, *, gamma: float = 1.4, time: float | None = None,
                   fmt: str = "auto", run: dict | None = None) -> Path:
    """Writes one snapshot.  fmt: "hdf5" (needs h5py), "raw", or "auto"
    (HDF5 when h5py is importable, else raw).  run: optional counters
    (step, cfl_max, offsets, dt; JSON-serialisable).  Returns the written path."""
    data = snapshot_arrays(U, rhs, gamma)
    path = Path(path)
    if fmt == "auto":
        try:
            import h5py  # noqa: F401
            fmt = "hdf5"
        except ImportError:
            fmt = "raw"
    if fmt == "hdf5":
        import h5py
        with h5py.File(path, "w") as f:
            for name in DATASETS:
                f.create_dataset(name, data=np.ascontiguousarray(data[name]))
            if time is not None:
                f.attrs["time"] = float(time)
            if run is not None:
                f.attrs["run"] = json.dumps(run)
        return path
    if fmt != "raw":
        raise ValueError(f"unknown snapshot format {fmt!r}")
    path.mkdir(parents=True, exist_ok=True)
    nx, ny = data["Rho"].shape
    for name in DATASETS:
        np.ascontiguousarray(data[name], dtype="<f8").tofile(path / f"{name}.f64")
    index = {"datasets": list(DATASETS), "shape": [nx, ny], "dtype": "float64 little-endian",
             "order": "x-major: value (i, j) at i * ny + j", "source": "Output::WriteToHDF5 layout"}
    if time is not None:
        index["time"] = float(time)
    if run is not None:
        index["run"] = run
    (path / "index.json").write_text(json.dumps(index, indent=1) + "\n")
    return path


def read_snapshot(path) -> dict[str, np.ndarray]:
    """Reads a snapshot written by write_snapshot (either format)."""
    path = Path(path)
    if path.is_dir():
        index = json.loads((path / "index.json").read_text())
        nx, ny = index["shape"]
        return {name: np.fromfile(path / f"{name}.f64", dtype="<f8").reshape(nx, ny) for name in index["datasets"]}
    import h5py
    with h5py.File(path, "r") as f:
        return {name: f[name][...] for name in DATASETS}


def read_run(path) -> dict:
    """The run counters (and time) stored with a snapshot, {} when it has none."""
    path = Path(path)
    if path.is_dir():
        index = json.loads((path / "index.json").read_text())
        run = dict(index.get("run", {}))
        if "time" in index:
            run["time"] = index["time"]
        return run
    import h5py
    with h5py.File(path, "r") as f:
        run = json.loads(f.attrs["run"]) if "run" in f.attrs else {}
        if "time" in f.attrs:
            run["time"] = float(f.attrs["time"])
    return run


def write_solver_snapshot(solver, path, *, time: float | None = None, dt: float | None = None,
                          fmt: str = "auto") -> Path:
    """Snapshot of an engine Solver: its state, its last RHS when it was
    created with keep_rhs=True (else the flux datasets are zero), and its run
    counters (Solver.run_counters) with the caller's time and last dt."""
    U = solver.get_state()
    rhs = solver.get_rhs() if solver.config.keep_rhs else None
    run = solver.run_counters()
    if dt is not None:
        run["dt"] = float(dt)
    return write_snapshot(path, U, rhs, gamma=solver.config.gamma, time=time, fmt=fmt, run=run)


def resume_solver(solver, path) -> dict:
    """Loads a snapshot written by write_solver_snapshot into a Solver of the
    same configuration so that its next steps are the bits the original run
    would have taken (storage offsets, state, step counter, carried CFL
    maximum).  Returns the stored run counters (with time and dt)."""
    d = read_snapshot(path)
    U = np.stack([d["Rho"], d["Mu"], d["Mv"], d["Energy"]])
    run = read_run(path)
    if not run:
        raise ValueError(f"{path} holds no run counters (written without them)")
    solver.resume(U, run)
    return run
