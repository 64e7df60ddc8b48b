"""cfs_compute_dt_static: the CFL step for callers that cannot allocate device
memory (a host code that owns all device memory through its own pool, or code
that must not allocate inside its time loop).  It takes a device state the
caller owns and must give the same dt, bit for bit, as the context-based
cfs_compute_dt on the same state -- on two calls in a row, since every call
reuses the same static scratch array.

This file is collected last on purpose; it runs alone in a fresh process or
after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_dt(cfsb, U_dev, types_dev, nx, ny, lx, ly, cfl, stream=None):
    lib = cfsb.load_library()
    dt = ctypes.c_double(0.0)
    rc = lib.cfs_compute_dt_static(ctypes.c_void_p(U_dev), ctypes.c_void_p(types_dev), nx, ny, lx, ly, 1.4, cfl,
                                   ctypes.c_void_p(stream), ctypes.byref(dt))
    if rc != 0:
        raise cfsb.CfsError(rc, lib.cfs_last_error(None).decode())
    return dt.value


def test_static_dt_matches_context_dt_twice(cfsb, workloads):
    import torch

    nx, ny = 300, 217
    w = workloads.riemann_quadrants(nx, ny, seed=12)
    with cfsb.Solver(nx, ny) as s:
        s.set_state(w.U0)
        ref = s.compute_dt(0.5)
    U_dev = torch.tensor(w.U0, dtype=torch.float64, device="cuda:0").contiguous()
    torch.cuda.synchronize()
    first = _static_dt(cfsb, U_dev.data_ptr(), 0, nx, ny, 1.0, 1.0, 0.5)
    second = _static_dt(cfsb, U_dev.data_ptr(), 0, nx, ny, 1.0, 1.0, 0.5)
    assert first == ref and second == ref


def test_static_dt_with_immersed_cells_and_a_stream(cfsb, workloads):
    import torch

    w = workloads.mach3_cylinder(256, 128)
    types, *_ = cfsb.circle_setup(256, 128, 2.0, 1.0, *w.circle, 400)
    U = w.U0.copy()
    U[:, types != 0] = 0.0  # solid cells hold zeros as in the reference (Run.cpp:98-104)
    with cfsb.Solver(256, 128, 2.0, 1.0, bc=w.bc, bc_prim=w.bc_prim) as s:
        s.build_circle(*w.circle, 400)
        s.set_state(U)
        ref = s.compute_dt(0.5)
    U_dev = torch.tensor(U, dtype=torch.float64, device="cuda:0").contiguous()
    t_dev = torch.tensor(types, dtype=torch.uint8, device="cuda:0").contiguous()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        got = _static_dt(cfsb, U_dev.data_ptr(), t_dev.data_ptr(), 256, 128, 2.0, 1.0, 0.5, stream.cuda_stream)
        assert got == ref


def test_static_dt_refuses_grids_beyond_its_scratch(cfsb):
    with pytest.raises(cfsb.CfsError) as e:
        # the size check comes before any device work, so no state is needed
        _static_dt(cfsb, 1 << 20, 0, 4097, 4096, 1.0, 1.0, 0.5)
    assert e.value.code == 1 and "static scratch limit" in str(e.value)


@pytest.mark.parametrize("nx,ny", [(4096, 1024), (4096, 4096)])
def test_static_dt_on_many_blocks_matches_context_dt(cfsb, workloads, nx, ny):
    """512 and 2048 partial blocks: the final kernel's strided loop over more
    than its 256 threads, and the largest grid the static scratch admits."""
    import torch

    w = workloads.riemann_quadrants(nx, ny, seed=13)
    with cfsb.Solver(nx, ny) as s:
        s.set_state(w.U0)
        ref = s.compute_dt(0.5)
    U_dev = torch.tensor(w.U0, dtype=torch.float64, device="cuda:0").contiguous()
    del w
    torch.cuda.synchronize()
    for _ in range(2):
        assert _static_dt(cfsb, U_dev.data_ptr(), 0, nx, ny, 1.0, 1.0, 0.5) == ref
    del U_dev
    torch.cuda.empty_cache()


def test_static_dt_reports_a_non_finite_cell(cfsb, workloads):
    import torch

    w = workloads.riemann_quadrants(300, 217, seed=12)
    U = w.U0.copy()
    U[3, 150, 100] = np.nan
    U_dev = torch.tensor(U, dtype=torch.float64, device="cuda:0").contiguous()
    torch.cuda.synchronize()
    with pytest.raises(cfsb.CfsError) as e:
        _static_dt(cfsb, U_dev.data_ptr(), 0, 300, 217, 1.0, 1.0, 0.5)
    assert e.value.code == 5
    # the shared scratch holds nothing over from the failed call
    U_dev[3, 150, 100] = float(w.U0[3, 150, 100])
    torch.cuda.synchronize()
    with cfsb.Solver(300, 217) as s:
        s.set_state(w.U0)
        assert _static_dt(cfsb, U_dev.data_ptr(), 0, 300, 217, 1.0, 1.0, 0.5) == s.compute_dt(0.5)
