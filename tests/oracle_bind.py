"""ctypes bindings of the checkers under oracle/ (test infrastructure only):

* ``oracle/_ref/libref_strict.so`` -- the reference solver's own classes, built
  from the reference tree against repo-written Eigen/MPI shims (oracle/Makefile);
* ``oracle/libcfs_oracle.so`` -- the C restatement (oracle/cfs_oracle.c).

Both take and return conserved states as float64 arrays of shape (4, nx, ny).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE = ROOT / "oracle"
REF_STRICT = ORACLE / "_ref" / "libref_strict.so"
REF_PERF = ORACLE / "_ref" / "libref_perf.so"
REF_GPU = ORACLE / "_ref" / "libref_gpu.so"
ORACLE_LIB = ORACLE / "libcfs_oracle.so"


def _reference_tree() -> Path | None:
    """The reference source tree, as oracle/Makefile resolves it
    (CFS_REFERENCE_TREE or the recipe's own default), or None when absent."""
    try:
        r = subprocess.run(["make", "-s", "-C", str(ORACLE), "ref-tree"], capture_output=True, text=True, timeout=60)
    except (OSError, subprocess.TimeoutExpired):
        return None
    out = r.stdout.strip()
    return Path(out) if r.returncode == 0 and out else None


REFERENCE_TREE = _reference_tree()

_dp = ctypes.POINTER(ctypes.c_double)


def P(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("integrator", ctypes.c_int), ("dt", ctypes.c_double), ("cfl", ctypes.c_double),
                ("bc_type", ctypes.c_int * 4), ("bc_prim", (ctypes.c_double * 4) * 4), ("circle", ctypes.c_int),
                ("radius", ctypes.c_double), ("cx", ctypes.c_double), ("cy", ctypes.c_double),
                ("npoints", ctypes.c_int)]


class OrcConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("gamma", ctypes.c_double), ("weno_eps", ctypes.c_double), ("rk", ctypes.c_int),
                ("hll", ctypes.c_int), ("bc", ctypes.c_int * 4), ("bc_U", (ctypes.c_double * 4) * 4),
                ("viscous", ctypes.c_int), ("mu", ctypes.c_double), ("prandtl", ctypes.c_double),
                ("mach", ctypes.c_double), ("nthreads", ctypes.c_int),
                ("positivity", ctypes.c_int)]


class OrcIB(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("cell", ctypes.c_void_p), ("donor", ctypes.c_void_p),
                ("image", ctypes.c_void_p), ("normal", ctypes.c_void_p), ("mode", ctypes.c_int),
                ("types", ctypes.c_void_p)]


def ensure_built() -> None:
    """Builds the checkers when missing (needs the reference tree for _ref)."""
    targets = []
    if not ORACLE_LIB.exists():
        targets.append("oracle")
    if (not REF_STRICT.exists() or not REF_PERF.exists()) and REFERENCE_TREE is not None:
        targets.append("ref")
    if targets:
        subprocess.run(["make", "-C", str(ORACLE), "-j8", *targets], check=True, capture_output=True)


_ref = None
_orc = None


def ref_lib(perf: bool = False) -> ctypes.CDLL:
    global _ref
    ensure_built()
    if perf:
        lib = ctypes.CDLL(str(REF_PERF))
        lib.ref_time_stages.restype = ctypes.c_double
        return lib
    if _ref is None:
        _ref = ctypes.CDLL(str(REF_STRICT))
        _ref.ref_time_stages.restype = ctypes.c_double
    return _ref


def orc_lib() -> ctypes.CDLL:
    global _orc
    ensure_built()
    if _orc is None:
        _orc = ctypes.CDLL(str(ORACLE_LIB))
        _orc.orc_cfl_dt.restype = ctypes.c_double
        _orc.orc_weno5.restype = ctypes.c_double
        _orc.orc_weno5.argtypes = [_dp, ctypes.c_double]
    return _orc


GAMMA = 1.4
RK_TVD2, RK_TVD3_REFERENCE, RK_SSP3 = 0, 1, 2


def dirichlet_conserved(prim, gamma: float = GAMMA):
    """Ghost state of DirichletBoundary with the Cylinder.cpp:22-32 body."""
    rho, u, v, p = prim
    mx, my = rho * u, rho * v
    return [rho, mx, my, p / (gamma - 1) + 0.5 * (mx * mx + my * my) / rho]


def make_ref_config(nx, ny, lx=1.0, ly=1.0, integrator=3, dt=1e-3, cfl=0.0, bc=(0, 0, 0, 0), bc_prim=None,
                    circle=None, npoints=400) -> RefConfig:
    c = RefConfig(nx=nx, ny=ny, lx=lx, ly=ly, integrator=integrator, dt=dt, cfl=cfl)
    for s in range(4):
        c.bc_type[s] = int(bc[s])
        prim = (bc_prim[s] if bc_prim is not None else (1.0, 0.0, 0.0, 1.0))
        for q in range(4):
            c.bc_prim[s][q] = prim[q]
    if circle is not None:
        c.circle = 1
        c.radius, c.cx, c.cy = circle
        c.npoints = npoints
    return c


def make_orc_config(nx, ny, lx=1.0, ly=1.0, rk=RK_TVD3_REFERENCE, hll=0, bc=(0, 0, 0, 0), bc_prim=None,
                    weno_eps=1e-2, viscous=0, mu=1e-3, prandtl=0.72, mach=1.0, nthreads=0,
                    positivity=0) -> OrcConfig:
    c = OrcConfig(nx=nx, ny=ny, lx=lx, ly=ly, gamma=GAMMA, weno_eps=weno_eps, rk=rk, hll=hll, viscous=viscous,
                  mu=mu, prandtl=prandtl, mach=mach, nthreads=nthreads, positivity=positivity)
    for s in range(4):
        c.bc[s] = int(bc[s])
        cons = dirichlet_conserved(bc_prim[s] if bc_prim is not None else (1.0, 0.0, 0.0, 1.0))
        for q in range(4):
            c.bc_U[s][q] = cons[q]
    return c


def ref_gpu_lib() -> ctypes.CDLL:
    """The reference's classes with the product's GPU plugins registered
    (oracle/Makefile target gpu; built where the reference tree is)."""
    return ctypes.CDLL(str(REF_GPU))


def ref_gpu_run(nx, ny, U0, nstages, precision=2, **kw):
    """The reference loop driven through the GPU plugins: returns the state."""
    c = make_ref_config(nx, ny, **kw)
    U0 = np.ascontiguousarray(U0, dtype=np.float64)
    out = np.zeros_like(U0)
    err = ctypes.create_string_buffer(512)
    rc = ref_gpu_lib().ref_gpu_run(ctypes.byref(c), P(U0), int(nstages), int(precision), P(out), err, 512)
    if rc != 0:
        raise RuntimeError(f"ref_gpu_run failed: {err.value.decode()}")
    return out


def ref_run(nx, ny, U0, nstages, **kw):
    """Reference run: returns (state, rhs, dt_log)."""
    c = make_ref_config(nx, ny, **kw)
    U0 = np.ascontiguousarray(U0, dtype=np.float64)
    out = np.zeros_like(U0)
    rhs = np.zeros_like(U0)
    dts = np.zeros(max(nstages, 1))
    ref_lib().ref_run(ctypes.byref(c), P(U0), int(nstages), P(out), P(rhs), P(dts))
    return out, rhs, dts[:nstages]


def ref_ib_info(nx, ny, lx, ly, circle, npoints=400, max_ig=200000):
    c = make_ref_config(nx, ny, lx=lx, ly=ly, circle=circle, npoints=npoints)
    types = np.zeros((nx, ny), np.int32)
    ig = np.zeros(2 * max_ig, np.int32)
    img = np.zeros(2 * max_ig)
    don = np.zeros(8 * max_ig, np.int32)
    nd = np.zeros(max_ig, np.int32)
    n = ref_lib().ref_ib_info(ctypes.byref(c), P(types), max_ig, P(ig), P(img), P(don), P(nd))
    assert n >= 0, "too many immersed-ghost cells"
    cells = (ig[0:2 * n:2] * ny + ig[1:2 * n:2]).astype(np.int32)
    d = don[:8 * n].reshape(n, 4, 2)
    donors = np.where(d[:, :, 0] >= 0, d[:, :, 0] * ny + d[:, :, 1], -1).astype(np.int32)
    return types.astype(np.uint8), cells, donors, img[:2 * n].reshape(n, 2).copy(), nd[:n].copy()


class OrcIBList:
    """Keeps the arrays of an OrcIB alive."""

    def __init__(self, cells, donors, images, normals=None, mode=0, types=None):
        self.types = None if types is None else np.ascontiguousarray(types, dtype=np.uint8).ravel()
        self.cells = np.ascontiguousarray(cells, dtype=np.int32)
        self.donors = np.ascontiguousarray(donors, dtype=np.int32).ravel()
        self.images = np.ascontiguousarray(images, dtype=np.float64).ravel()
        n = self.cells.size
        self.normals = (np.zeros(2 * n) if normals is None
                        else np.ascontiguousarray(normals, dtype=np.float64).ravel())
        self.s = OrcIB(n=n, cell=self.cells.ctypes.data, donor=self.donors.ctypes.data,
                       image=self.images.ctypes.data, normal=self.normals.ctypes.data, mode=mode,
                       types=None if self.types is None else self.types.ctypes.data)


def orc_run(cfg: OrcConfig, U0, first, count, dt=1e-3, cfl=0.0, types=None, ib: OrcIBList | None = None):
    """Oracle run over loop counters first..first+count-1; returns (state, dt_log)."""
    U = np.ascontiguousarray(U0, dtype=np.float64).copy()
    t = (np.zeros(cfg.nx * cfg.ny, np.uint8) if types is None
         else np.ascontiguousarray(types, dtype=np.uint8).ravel())
    ibs = ib.s if ib is not None else OrcIB(n=0)
    dts = np.zeros(max(count, 1))
    orc_lib().orc_run(ctypes.byref(cfg), P(t), ctypes.byref(ibs), P(U), int(first), int(count),
                      ctypes.c_double(dt), ctypes.c_double(cfl), P(dts))
    return U, dts[:count]


def orc_stage(cfg: OrcConfig, U, U0, U1, stage, dt, types=None, ib: OrcIBList | None = None, rhs=None):
    """One oracle stage in place on U (U0/U1 are the stage copies)."""
    t = (np.zeros(cfg.nx * cfg.ny, np.uint8) if types is None
         else np.ascontiguousarray(types, dtype=np.uint8).ravel())
    ibs = ib.s if ib is not None else OrcIB(n=0)
    orc_lib().orc_stage(ctypes.byref(cfg), P(t), ctypes.byref(ibs), int(stage), ctypes.c_double(dt), P(U), P(U0),
                        P(U1), None if rhs is None else P(rhs))


def orc_cfl_dt(cfg: OrcConfig, U, cfl, types=None) -> float:
    t = None if types is None else np.ascontiguousarray(types, dtype=np.uint8).ravel()
    U = np.ascontiguousarray(U, dtype=np.float64)
    return orc_lib().orc_cfl_dt(ctypes.byref(cfg), None if t is None else P(t), P(U), ctypes.c_double(cfl))


def stage_of(rk: int, counter: int) -> int:
    if rk == RK_TVD2:
        return 1 if counter % 2 == 0 else 0
    return 2 if counter % 3 == 0 else (0 if counter % 3 == 1 else 1)
