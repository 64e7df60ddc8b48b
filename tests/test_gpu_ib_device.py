"""On-device circle set-up (cfs_circle_setup_device, cfs_ib_build_circle_device)
against the host set-up, which is pinned to the reference's own classes: cell
types, the ghost list, image points and normals are bit for bit equal (the
kernels are built without FMA contraction), and so are the host-chosen donors;
a solver set up either way takes the same steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, lx, ly, r, cx, cy
    (2048, 1024, 2.0, 1.0, 0.05, 0.4, 0.5),    # the Mach-3 cylinder grid
    (256, 128, 2.0, 1.0, 0.05, 0.4, 0.5),
    (300, 200, 1.0, 1.0, 0.2, 0.5, 0.5),
    (128, 160, 1.0, 1.0, 0.08, 0.13, 0.77),
    (97, 64, 1.0, 1.0, 0.3, 0.95, 0.5),         # body cut by the right side
]


def _random_cases(n, seed=5):
    rng = np.random.default_rng(seed)
    edges = np.arange(64, 769, 16)
    out = []
    for _ in range(n):
        nx, ny = int(rng.choice(edges)), int(rng.choice(edges))
        r = rng.uniform(0.03, 0.1)
        out.append((nx, ny, 1.0, 1.0, r, rng.uniform(3 * r, 1 - 3 * r), rng.uniform(3 * r, 1 - 3 * r)))
    return out


@pytest.mark.parametrize("case", CASES + _random_cases(12))
def test_device_setup_is_the_host_setup(cfsb, case):
    nx, ny, lx, ly, r, cx, cy = case
    try:
        host = cfsb.circle_setup(nx, ny, lx, ly, r, cx, cy, 400)
    except cfsb.CfsError as e:  # too few fluid donors: the device set-up refuses alike
        with pytest.raises(cfsb.CfsError) as d:
            cfsb.circle_setup(nx, ny, lx, ly, r, cx, cy, 400, device=0)
        assert str(d.value) == str(e)
        return
    dev = cfsb.circle_setup(nx, ny, lx, ly, r, cx, cy, 400, device=0)
    for name, a, b in zip(("types", "cells", "donors", "images", "normals"), host, dev):
        assert a.shape == b.shape, name
        assert np.array_equal(a, b), (name, case)
    assert host[1].size > 0


def test_solver_set_up_on_device_steps_alike(cfsb, workloads):
    w = workloads.mach3_cylinder(256, 128)
    out = []
    for on_device in (False, True):
        with cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=w.bc,
                         bc_prim=w.bc_prim, positivity=cfsb.POSITIVITY_BODY) as s:
            s.build_circle(*w.circle, 400, cfsb.IB_BILINEAR_SLIP, on_device=on_device)
            ib = s.get_ib()
            s.set_state(w.U0)
            s.advance(20, cfl=0.5)
            out.append((ib, s.get_state()))
    (ib0, U0), (ib1, U1) = out
    for a, b in zip(ib0, ib1):
        assert np.array_equal(a, b)
    assert np.array_equal(U0, U1)
