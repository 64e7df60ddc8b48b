"""The reference program's own loop with the GPU plugins registered at its
plugin selection point (2d_compressible_flow_solver_b200/adapter, the drop-in
at Run.cpp:41-48): in the FP64_EXACT form the run must equal the unmodified
reference's run bit for bit, NaN positions included."""
import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

MACH3 = (1.4, 3.0, 0.0, 1.0)


def _needs_gpu_harness():
    if not ob.REF_GPU.exists():
        pytest.skip("oracle/_ref/libref_gpu.so not built (needs the reference tree at build time)")


@pytest.mark.parametrize("integrator", [2, 3])
def test_plugins_reproduce_reference_loop_quadrants(workloads, integrator):
    _needs_gpu_harness()
    w = workloads.riemann_quadrants(64, 48, seed=4)
    kw = dict(lx=1.0, ly=1.0, integrator=integrator, dt=1e-3)
    ref, _, _ = ob.ref_run(64, 48, w.U0, 12, **kw)
    got = ob.ref_gpu_run(64, 48, w.U0, 12, precision=2, **kw)
    assert np.isfinite(ref).mean() > 0.9
    assert np.array_equal(got, ref, equal_nan=True)


def test_plugins_reproduce_reference_loop_with_circle(workloads):
    _needs_gpu_harness()
    nx, ny = 96, 64
    # the reference's own cylinder set-up (Cylinder.cpp: rho 1, u 1, p 1 inflow)
    prim = (1.0, 1.0, 0.0, 1.0)
    U = workloads.conserved(np.full((nx, ny), prim[0]), prim[1], prim[2], prim[3])
    kw = dict(lx=1.5, ly=1.0, integrator=2, dt=5e-4, bc=(1, 0, 0, 0), bc_prim=[prim] * 4, circle=(0.12, 0.5, 0.5))
    ref, _, _ = ob.ref_run(nx, ny, U, 10, **kw)
    got = ob.ref_gpu_run(nx, ny, U, 10, precision=2, **kw)
    assert np.all(np.isfinite(ref))
    assert np.array_equal(got, ref)
