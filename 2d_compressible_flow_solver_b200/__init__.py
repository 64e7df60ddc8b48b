"""B200 (sm_100a) stage engine for the 2-D compressible-flow solver.

Python binding, through ctypes, of the C ABI in ``include/cfs.h`` implemented by
``libcfs.so`` (built in this folder by ``build.py``).  The binding holds no
numerics: every call goes to the CUDA library, and there is no CPU fallback --
creating a :class:`Solver` without a CUDA device raises :class:`CfsError`.

Arrays use the reference solver's cell order ``U[v, i, j]`` with
``v = (rho, rho*u, rho*v, E)``, ``i`` the x index and ``j`` the y index
(``cells[i][j]`` in source/meshes/CartesianMesh.cpp:3-9).

The package folder's name starts with a digit, so import it with
``importlib.import_module("2d_compressible_flow_solver_b200")``.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

__all__ = [
    "LIB_PATH", "CfsConfig", "CfsCase", "CfsError", "Solver", "Batch", "load_library", "exported_symbols", "circle_setup",
    "polygon_setup",
    "FP64", "FP32_MIXED", "FP64_EXACT", "RK_TVD2", "RK_TVD3_REFERENCE", "RK_SSP3",
    "HLL_REFERENCE", "HLL_DAVIS", "BC_NEUMANN", "BC_DIRICHLET", "BC_PERIODIC", "BC_HALO",
    "CELL_FLUID", "CELL_SOLID", "CELL_IMMERSED_GHOST", "IB_REFERENCE", "IB_BILINEAR_SLIP",
    "VISCOUS_OFF", "VISCOUS_NS", "POSITIVITY_OFF", "POSITIVITY_FACE", "POSITIVITY_BODY", "POSITIVITY_FLOOR", "ROUND_STOCHASTIC",
    "ROUND_NEAREST", "ROUND_STOCHASTIC_ALL", "PART_ALL", "PART_INTERIOR", "PART_EDGES", "variants", "fp_peaks",
]

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libcfs.so"
HEADER_PATH = _HERE.parent / "include" / "cfs.h"

FP64, FP32_MIXED, FP64_EXACT = 0, 1, 2
RK_TVD2, RK_TVD3_REFERENCE, RK_SSP3 = 0, 1, 2
HLL_REFERENCE, HLL_DAVIS = 0, 1
BC_NEUMANN, BC_DIRICHLET, BC_PERIODIC, BC_HALO = 0, 1, 2, 3
CELL_FLUID, CELL_SOLID, CELL_IMMERSED_GHOST = 0, 1, 2
IB_REFERENCE, IB_BILINEAR_SLIP = 0, 1
VISCOUS_OFF, VISCOUS_NS = 0, 1
POSITIVITY_OFF, POSITIVITY_FACE, POSITIVITY_BODY, POSITIVITY_FLOOR = 0, 1, 2, 3
ROUND_STOCHASTIC, ROUND_NEAREST, ROUND_STOCHASTIC_ALL = 0, 1, 2
PART_ALL, PART_INTERIOR, PART_EDGES = 0, 1, 2

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int32_p = ctypes.POINTER(ctypes.c_int32)
_c_uint8_p = ctypes.POINTER(ctypes.c_uint8)


class CfsConfig(ctypes.Structure):
    """Mirror of ``struct cfs_config`` (include/cfs.h)."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("gamma", ctypes.c_double), ("weno_eps", ctypes.c_double),
        ("precision", ctypes.c_int), ("rk", ctypes.c_int), ("hll", ctypes.c_int),
        ("bc", ctypes.c_int * 4), ("bc_prim", (ctypes.c_double * 4) * 4),
        ("viscous", ctypes.c_int),
        ("mu", ctypes.c_double), ("prandtl", ctypes.c_double), ("mach", ctypes.c_double),
        ("keep_rhs", ctypes.c_int), ("device", ctypes.c_int), ("variant", ctypes.c_int),
        ("positivity", ctypes.c_int), ("rounding", ctypes.c_int), ("march_rows", ctypes.c_int),
    ]


class CfsCase(ctypes.Structure):
    """Mirror of ``struct cfs_case`` (include/cfs.h)."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("bc", ctypes.c_int * 4), ("bc_prim", (ctypes.c_double * 4) * 4),
        ("circle", ctypes.c_int), ("radius", ctypes.c_double), ("cx", ctypes.c_double), ("cy", ctypes.c_double),
        ("npoints", ctypes.c_int), ("ib_mode", ctypes.c_int), ("rows", ctypes.c_int), ("edge_code", ctypes.c_int),
    ]


class CfsError(RuntimeError):
    """A cfs_* call returned a non-zero status; ``code`` is that status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"cfs error {code}: {message}")
        self.code = code


_lib = None

# name -> (restype, argtypes), one entry per declaration of include/cfs.h
_SIGNATURES = {
    "cfs_abi_version": (ctypes.c_int, []),
    "cfs_variant_count": (ctypes.c_int, []),
    "cfs_variant_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "cfs_config_default": (None, [ctypes.POINTER(CfsConfig)]),
    "cfs_create": (ctypes.c_int, [ctypes.POINTER(CfsConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "cfs_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cfs_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cfs_set_state": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_get_state": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_get_rhs": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_set_cell_types": (ctypes.c_int, [ctypes.c_void_p, _c_uint8_p]),
    "cfs_set_ib": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_int32_p, _c_int32_p,
                                  _c_double_p, _c_double_p]),
    "cfs_ib_build_circle": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_int]),
    "cfs_circle_setup": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _c_uint8_p,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_int), _c_int32_p, _c_int32_p,
                                        _c_double_p, _c_double_p]),
    "cfs_ib_build_circle_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "cfs_circle_setup_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_int, _c_uint8_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                               _c_int32_p, _c_int32_p, _c_double_p, _c_double_p]),
    "cfs_ib_build_polygon": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p, ctypes.c_int]),
    "cfs_polygon_setup": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                         _c_double_p, _c_uint8_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         _c_int32_p, _c_int32_p, _c_double_p, _c_double_p]),
    "cfs_get_ib": (ctypes.c_int, [ctypes.c_void_p, _c_uint8_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                  _c_int32_p, _c_int32_p, _c_double_p]),
    "cfs_ib_fill": (ctypes.c_int, [ctypes.c_void_p]),
    "cfs_compute_dt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _c_double_p]),
    "cfs_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]),
    "cfs_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cfs_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   _c_double_p, _c_double_p]),
    "cfs_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "cfs_get_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "cfs_halo_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "cfs_halo_pack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "cfs_halo_unpack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "cfs_set_storage_offsets": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_steps_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]),
    "cfs_steps_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cfs_cfl_export": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cfs_cfl_import": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cfs_steps_end": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "cfs_get_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint), _c_double_p, _c_double_p]),
    "cfs_set_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint, ctypes.c_double]),
    "cfs_conserved_totals": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_compute_dt_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_void_p, _c_double_p]),
    "cfs_fp_peaks": (ctypes.c_int, [ctypes.c_int, _c_double_p, _c_double_p, _c_double_p]),
    "cfs_batch_create": (ctypes.c_int, [ctypes.POINTER(CfsConfig), ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "cfs_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cfs_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cfs_batch_set_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "cfs_batch_get_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "cfs_batch_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         _c_double_p]),
    "cfs_batch_get_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "cfs_batch_advance_dt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p, _c_double_p]),
    "cfs_batch_dt_last": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "cfs_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_int)]),
    "cfs_weno5_faces": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p, _c_double_p, _c_double_p]),
    "cfs_hll_faces": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p,
                                     _c_double_p]),
}


def load_library() -> ctypes.CDLL:
    """Loads libcfs.so once and declares every entry point's signature.

    Raises ImportError when the library has not been built (run build.py).
    """
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run python {_HERE / 'build.py'}")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def variants() -> list[tuple[int, int, int, int]]:
    """(rows, warps, min_blocks, load schedule) of every stage-kernel variant, index v-1."""
    lib = load_library()
    out = []
    for v in range(1, lib.cfs_variant_count() + 1):
        r, w, b, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib.cfs_variant_info(v, ctypes.byref(r), ctypes.byref(w), ctypes.byref(b), ctypes.byref(p))
        out.append((r.value, w.value, b.value, p.value))
    return out


def fp_peaks(device: int = 0) -> dict:
    """Measured CUDA-core peaks of a device (cfs_fp_peaks), TFLOP/s."""
    lib = load_library()
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    rc = lib.cfs_fp_peaks(int(device), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    if rc != 0:
        raise CfsError(rc, lib.cfs_last_error(None).decode())
    return {"fp32_ffma": a.value, "fp32_ffma2": b.value, "fp64_dfma": c.value}


def exported_symbols() -> list[str]:
    """Names of the entry points this binding declares (all of include/cfs.h)."""
    return list(_SIGNATURES)


def circle_setup(nx: int, ny: int, lx: float, ly: float, radius: float, cx: float, cy: float, npoints: int = 400,
                 device: int | None = None):
    """Circle immersed-boundary set-up: returns (types[nx, ny], cells[n],
    donors[n, 4], images[n, 2], normals[n, 2]).  device=None: the host set-up
    (cfs_circle_setup); an ordinal: the per-cell work on that GPU
    (cfs_circle_setup_device), bit for bit the same result."""
    lib = load_library()
    types = np.empty((nx, ny), dtype=np.uint8)
    n = ctypes.c_int(0)
    args = (int(nx), int(ny), float(lx), float(ly), float(radius), float(cx), float(cy), int(npoints))
    if device is None:
        call = lib.cfs_circle_setup
    else:
        def call(*a):
            return lib.cfs_circle_setup_device(int(device), *a)
    rc = call(*args, types.ctypes.data_as(_c_uint8_p), 0, ctypes.byref(n), None, None, None, None)
    if rc != 0:
        raise CfsError(rc, lib.cfs_last_error(None).decode())
    cells = np.empty(n.value, dtype=np.int32)
    donors = np.empty((n.value, 4), dtype=np.int32)
    images = np.empty((n.value, 2))
    normals = np.empty((n.value, 2))
    rc = call(*args, None, n.value, ctypes.byref(n), cells.ctypes.data_as(_c_int32_p),
              donors.ctypes.data_as(_c_int32_p), images.ctypes.data_as(_c_double_p), normals.ctypes.data_as(_c_double_p))
    if rc != 0:
        raise CfsError(rc, lib.cfs_last_error(None).decode())
    return types, cells, donors, images, normals


def polygon_setup(nx: int, ny: int, lx: float, ly: float, xy):
    """Host set-up of a closed polygon body (cfs_polygon_setup), vertices
    xy[npoints, 2] in order: returns (types[nx, ny], cells[n], donors[n, 4],
    images[n, 2], normals[n, 2])."""
    lib = load_library()
    v = np.ascontiguousarray(np.asarray(xy, dtype=np.float64).reshape(-1, 2))
    types = np.empty((nx, ny), dtype=np.uint8)
    n = ctypes.c_int(0)
    args = (int(nx), int(ny), float(lx), float(ly), int(v.shape[0]), v.ctypes.data_as(_c_double_p))
    rc = lib.cfs_polygon_setup(*args, types.ctypes.data_as(_c_uint8_p), 0, ctypes.byref(n), None, None, None, None)
    if rc != 0:
        raise CfsError(rc, lib.cfs_last_error(None).decode())
    cells = np.empty(n.value, dtype=np.int32)
    donors = np.empty((n.value, 4), dtype=np.int32)
    images = np.empty((n.value, 2))
    normals = np.empty((n.value, 2))
    rc = lib.cfs_polygon_setup(*args, None, n.value, ctypes.byref(n), cells.ctypes.data_as(_c_int32_p),
                               donors.ctypes.data_as(_c_int32_p), images.ctypes.data_as(_c_double_p),
                               normals.ctypes.data_as(_c_double_p))
    if rc != 0:
        raise CfsError(rc, lib.cfs_last_error(None).decode())
    return types, cells, donors, images, normals


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_c_double_p)


class Solver:
    """One device-resident grid and its stage engine (a ``cfs_ctx``)."""

    def __init__(self, nx: int, ny: int, lx: float = 1.0, ly: float = 1.0, *, precision: int = FP64,
                 rk: int = RK_TVD3_REFERENCE, hll: int = HLL_REFERENCE, bc=(BC_NEUMANN,) * 4, bc_prim=None,
                 gamma: float = 1.4, weno_eps: float = 1e-2, viscous: int = VISCOUS_OFF, mu: float = 1e-3,
                 prandtl: float = 0.72, mach: float = 1.0, keep_rhs: bool = False, device: int = 0,
                 variant: int = 0, positivity: int = 0, rounding: int = ROUND_STOCHASTIC_ALL, march_rows: int = 0):
        self._lib = load_library()
        cfg = CfsConfig()
        self._lib.cfs_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny, cfg.lx, cfg.ly = int(nx), int(ny), float(lx), float(ly)
        cfg.gamma, cfg.weno_eps = float(gamma), float(weno_eps)
        cfg.precision, cfg.rk, cfg.hll = int(precision), int(rk), int(hll)
        for s in range(4):
            cfg.bc[s] = int(bc[s])
            if bc_prim is not None:
                for q in range(4):
                    cfg.bc_prim[s][q] = float(bc_prim[s][q])
        cfg.viscous, cfg.mu, cfg.prandtl, cfg.mach = int(viscous), float(mu), float(prandtl), float(mach)
        cfg.keep_rhs, cfg.device, cfg.variant = int(bool(keep_rhs)), int(device), int(variant)
        cfg.positivity, cfg.rounding, cfg.march_rows = int(positivity), int(rounding), int(march_rows)
        self.config = cfg
        self.nx, self.ny = int(nx), int(ny)
        self._ctx = ctypes.c_void_p()
        rc = self._lib.cfs_create(ctypes.byref(cfg), ctypes.byref(self._ctx))
        if rc != 0:
            raise CfsError(rc, self._lib.cfs_last_error(None).decode())

    # -- plumbing
    def _check(self, rc: int) -> None:
        if rc != 0:
            raise CfsError(rc, self._lib.cfs_last_error(self._ctx).decode())

    def _state_array(self, U) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (4, self.nx, self.ny):
            raise ValueError(f"state must have shape (4, {self.nx}, {self.ny}), got {U.shape}")
        return U

    def close(self) -> None:
        if self._ctx:
            self._lib.cfs_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state
    def set_state(self, U) -> None:
        U = self._state_array(U)
        self._check(self._lib.cfs_set_state(self._ctx, _dp(U)))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((4, self.nx, self.ny), dtype=np.float64)
        self._check(self._lib.cfs_get_state(self._ctx, _dp(out)))
        return out

    def get_rhs(self) -> np.ndarray:
        out = np.empty((4, self.nx, self.ny), dtype=np.float64)
        self._check(self._lib.cfs_get_rhs(self._ctx, _dp(out)))
        return out

    # -- immersed boundary
    def set_cell_types(self, types) -> None:
        t = np.ascontiguousarray(types, dtype=np.uint8).reshape(self.nx, self.ny)
        self._check(self._lib.cfs_set_cell_types(self._ctx, t.ctypes.data_as(_c_uint8_p)))

    def set_ib(self, mode: int, cells, donors, images, normals=None) -> None:
        cells = np.ascontiguousarray(cells, dtype=np.int32).ravel()
        donors = np.ascontiguousarray(donors, dtype=np.int32).ravel()
        images = np.ascontiguousarray(images, dtype=np.float64).ravel()
        n = cells.size
        nrm = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64).ravel()
        self._check(self._lib.cfs_set_ib(self._ctx, int(mode), n, cells.ctypes.data_as(_c_int32_p),
                                         donors.ctypes.data_as(_c_int32_p), _dp(images),
                                         None if nrm is None else _dp(nrm)))

    def build_circle(self, radius: float, cx: float, cy: float, npoints: int = 400, mode: int = IB_REFERENCE,
                     on_device: bool = False) -> None:
        """Circle immersed boundary (cfs_ib_build_circle; on_device: the per-cell
        set-up on the GPU, cfs_ib_build_circle_device, the same result)."""
        fn = self._lib.cfs_ib_build_circle_device if on_device else self._lib.cfs_ib_build_circle
        self._check(fn(self._ctx, radius, cx, cy, int(npoints), int(mode)))

    def build_polygon(self, xy, mode: int = IB_BILINEAR_SLIP) -> None:
        """Closed polygon body (cfs_ib_build_polygon), vertices xy[npoints, 2] in order."""
        v = np.ascontiguousarray(np.asarray(xy, dtype=np.float64).reshape(-1, 2))
        self._check(self._lib.cfs_ib_build_polygon(self._ctx, int(v.shape[0]), v.ctypes.data_as(_c_double_p), int(mode)))

    def get_ib(self):
        """Returns (types[nx, ny], cells[n], donors[n, 4], images[n, 2])."""
        types = np.empty((self.nx, self.ny), dtype=np.uint8)
        n = ctypes.c_int(0)
        self._check(self._lib.cfs_get_ib(self._ctx, types.ctypes.data_as(_c_uint8_p), 0, ctypes.byref(n),
                                         None, None, None))
        cells = np.empty(n.value, dtype=np.int32)
        donors = np.empty((n.value, 4), dtype=np.int32)
        images = np.empty((n.value, 2), dtype=np.float64)
        self._check(self._lib.cfs_get_ib(self._ctx, None, n.value, ctypes.byref(n),
                                         cells.ctypes.data_as(_c_int32_p), donors.ctypes.data_as(_c_int32_p),
                                         _dp(images)))
        return types, cells, donors, images

    def ib_fill(self) -> None:
        self._check(self._lib.cfs_ib_fill(self._ctx))

    # -- time stepping
    def compute_dt(self, cfl: float) -> float:
        dt = ctypes.c_double(0.0)
        self._check(self._lib.cfs_compute_dt(self._ctx, float(cfl), ctypes.byref(dt)))
        return dt.value

    def stage(self, counter: int, dt: float) -> None:
        self._check(self._lib.cfs_stage(self._ctx, int(counter), float(dt)))

    def step(self, dt: float) -> None:
        self._check(self._lib.cfs_step(self._ctx, float(dt)))

    def advance(self, nsteps: int, cfl: float = 0.0, dt: float = 0.0):
        """Runs nsteps RK steps; returns (simulated time advanced, last dt)."""
        t = ctypes.c_double(0.0)
        dl = ctypes.c_double(0.0)
        self._check(self._lib.cfs_advance(self._ctx, int(nsteps), float(cfl), float(dt), ctypes.byref(t),
                                          ctypes.byref(dl)))
        return t.value, dl.value

    def synchronize(self) -> None:
        self._check(self._lib.cfs_synchronize(self._ctx))

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        return int(self._lib.cfs_get_stream(self._ctx) or 0)

    def set_storage_offsets(self, off=None) -> None:
        """Fix the FP32-mixed storage offsets (4 values) for later set_state
        calls; None returns to the state's own means."""
        if off is None:
            self._check(self._lib.cfs_set_storage_offsets(self._ctx, None))
        else:
            a = np.ascontiguousarray(off, dtype=np.float64)
            if a.shape != (4,):
                raise ValueError("need 4 offsets")
            self._check(self._lib.cfs_set_storage_offsets(self._ctx, _dp(a)))

    def run_counters(self) -> dict:
        """Counters a bit-exact resume needs (cfs_get_step): completed steps,
        the carried CFL maximum (0 if none) and the FP32 storage offsets."""
        step = ctypes.c_uint(0)
        m = ctypes.c_double(0.0)
        off = np.zeros(4)
        self._check(self._lib.cfs_get_step(self._ctx, ctypes.byref(step), ctypes.byref(m), _dp(off)))
        return {"step": int(step.value), "cfl_max": float(m.value), "offsets": [float(x) for x in off]}

    def resume(self, U, counters: dict) -> None:
        """Installs a state and the counters of run_counters(), so that the
        following steps are those of the run the counters were taken from:
        storage offsets (FP32-mixed), state, then step and CFL maximum."""
        if self.config.precision == FP32_MIXED:
            self.set_storage_offsets(counters["offsets"])
        self.set_state(U)
        self._check(self._lib.cfs_set_step(self._ctx, int(counters["step"]), float(counters["cfl_max"])))

    # -- device-ordered stepping (decomposed grids): see cfs_steps_* in cfs.h
    def steps_begin(self, cfl: float = 0.0, dt: float = 0.0) -> None:
        self._check(self._lib.cfs_steps_begin(self._ctx, float(cfl), float(dt)))

    def steps_stage(self, part: int = PART_ALL) -> None:
        self._check(self._lib.cfs_steps_stage(self._ctx, int(part)))

    def cfl_export(self, dev_ptr: int) -> None:
        self._check(self._lib.cfs_cfl_export(self._ctx, ctypes.c_void_p(dev_ptr)))

    def cfl_import(self, dev_ptr: int) -> None:
        self._check(self._lib.cfs_cfl_import(self._ctx, ctypes.c_void_p(dev_ptr)))

    def steps_end(self):
        """Waits for the run of steps; returns (simulated time, last dt)."""
        t = ctypes.c_double(0.0)
        dl = ctypes.c_double(0.0)
        self._check(self._lib.cfs_steps_end(self._ctx, ctypes.byref(t), ctypes.byref(dl)))
        return t.value, dl.value

    def halo_bytes(self) -> int:
        n = ctypes.c_longlong(0)
        self._check(self._lib.cfs_halo_bytes(self._ctx, ctypes.byref(n)))
        return n.value

    def halo_pack(self, side: int, dev_ptr: int) -> None:
        self._check(self._lib.cfs_halo_pack(self._ctx, int(side), ctypes.c_void_p(dev_ptr)))

    def halo_unpack(self, side: int, dev_ptr: int) -> None:
        self._check(self._lib.cfs_halo_unpack(self._ctx, int(side), ctypes.c_void_p(dev_ptr)))

    def totals(self) -> np.ndarray:
        out = np.zeros(4, dtype=np.float64)
        self._check(self._lib.cfs_conserved_totals(self._ctx, _dp(out)))
        return out

    # -- unit-level batches
    def weno5_faces(self, stencils):
        """stencils[n, 6, 4] -> (left[n, 5], right[n, 5]) = (rho, mx, my, E, p)."""
        st = np.ascontiguousarray(stencils, dtype=np.float64)
        n = st.shape[0]
        left = np.empty((n, 5))
        right = np.empty((n, 5))
        self._check(self._lib.cfs_weno5_faces(self._ctx, n, _dp(st), _dp(left), _dp(right)))
        return left, right

    def hll_faces(self, direction: int, L, R) -> np.ndarray:
        L = np.ascontiguousarray(L, dtype=np.float64)
        R = np.ascontiguousarray(R, dtype=np.float64)
        F = np.empty_like(L)
        self._check(self._lib.cfs_hll_faces(self._ctx, L.shape[0], int(direction), _dp(L), _dp(R), _dp(F)))
        return F


class Batch:
    """Many independent grids advanced together (a ``cfs_batch``): one
    persistent launch per stage for all cases, per-case CFL dt on the device.
    A case without ``rows`` takes the work-unit rows the autotuner measured
    best for its size (``tuning.json`` ``batch_rows``; ``tuned_rows=False``:
    the library default)."""

    def __init__(self, cases, *, precision: int = FP32_MIXED, rk: int = RK_SSP3, hll: int = HLL_DAVIS,
                 gamma: float = 1.4, weno_eps: float = 1e-2, device: int = 0, positivity: int = POSITIVITY_OFF,
                 rounding: int = ROUND_STOCHASTIC_ALL, tuned_rows: bool = True):
        from . import autotune as _autotune
        self._lib = load_library()
        cfg = CfsConfig()
        self._lib.cfs_config_default(ctypes.byref(cfg))
        cfg.precision, cfg.rk, cfg.hll, cfg.gamma, cfg.weno_eps, cfg.device = (
            int(precision), int(rk), int(hll), float(gamma), float(weno_eps), int(device))
        cfg.positivity, cfg.rounding = int(positivity), int(rounding)
        arr = (CfsCase * len(cases))()
        self.shapes = []
        for k, c in enumerate(cases):
            d = arr[k]
            d.nx, d.ny, d.lx, d.ly = int(c["nx"]), int(c["ny"]), float(c.get("lx", 1.0)), float(c.get("ly", 1.0))
            for s in range(4):
                d.bc[s] = int(c.get("bc", (BC_NEUMANN,) * 4)[s])
                prim = c.get("bc_prim", [[1.0, 0.0, 0.0, 1.0]] * 4)[s]
                for q in range(4):
                    d.bc_prim[s][q] = float(prim[q])
            circle = c.get("circle")
            if circle is not None:
                d.circle = 1
                d.radius, d.cx, d.cy = (float(x) for x in circle)
                d.npoints = int(c.get("npoints", 400))
                d.ib_mode = int(c.get("ib_mode", IB_BILINEAR_SLIP))
            d.rows = int(c.get("rows", 0))
            if d.rows == 0 and tuned_rows:
                d.rows = _autotune.batch_rows_for("f32" if precision == FP32_MIXED else "f64", d.nx, d.ny)
            d.edge_code = int(bool(c.get("edge_code", False)))
            self.shapes.append((d.nx, d.ny))
        self._b = ctypes.c_void_p()
        rc = self._lib.cfs_batch_create(ctypes.byref(cfg), len(cases), ctypes.cast(arr, ctypes.c_void_p),
                                        ctypes.byref(self._b))
        if rc != 0:
            raise CfsError(rc, self._lib.cfs_batch_last_error(None).decode())

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise CfsError(rc, self._lib.cfs_batch_last_error(self._b).decode())

    def close(self) -> None:
        if self._b:
            self._lib.cfs_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        """The batch's cudaStream_t as an integer handle."""
        return int(self._lib.cfs_batch_get_stream(self._b) or 0)

    def info(self):
        cells = ctypes.c_longlong(0)
        items = ctypes.c_int(0)
        self._check(self._lib.cfs_batch_info(self._b, ctypes.byref(cells), ctypes.byref(items)))
        return cells.value, items.value

    def set_state(self, case: int, U) -> None:
        nx, ny = self.shapes[case]
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (4, nx, ny):
            raise ValueError(f"case {case}: state must have shape (4, {nx}, {ny})")
        self._check(self._lib.cfs_batch_set_state(self._b, int(case), _dp(U)))

    def get_state(self, case: int) -> np.ndarray:
        nx, ny = self.shapes[case]
        out = np.empty((4, nx, ny))
        self._check(self._lib.cfs_batch_get_state(self._b, int(case), _dp(out)))
        return out

    def advance(self, nsteps: int, cfl: float = 0.0, dt=0.0) -> np.ndarray:
        """Runs nsteps RK steps of every case (per-case CFL dt when cfl > 0;
        else dt, a common value or one per case); returns each case's
        simulated time."""
        t = np.zeros(len(self.shapes))
        if np.ndim(dt) == 0:
            self._check(self._lib.cfs_batch_advance(self._b, int(nsteps), float(cfl), float(dt), _dp(t)))
        else:
            d = np.ascontiguousarray(dt, dtype=np.float64)
            if d.shape != (len(self.shapes),):
                raise ValueError("need one dt per case")
            self._check(self._lib.cfs_batch_advance_dt(self._b, int(nsteps), _dp(d), _dp(t)))
        return t

    def dt_last(self) -> np.ndarray:
        """Per case, the dt of the last step taken."""
        d = np.zeros(len(self.shapes))
        self._check(self._lib.cfs_batch_dt_last(self._b, _dp(d)))
        return d


