"""The synthetic inputs stand in for the configurations' workloads: their
shapes, value ranges and seeded draws follow the configurations' statements
(four-quadrant states, smooth advection, Mach-3 cylinder, shear layer, the
uneven 512-case batch).  CPU only."""
import math

import numpy as np

GAMMA = 1.4


def _prim(U):
    rho = U[0]
    u, v = U[1] / rho, U[2] / rho
    p = (GAMMA - 1) * (U[3] - 0.5 * rho * (u * u + v * v))
    return rho, u, v, p


def test_four_quadrant_state(workloads):
    w = workloads.riemann_quadrants(256, 256, seed=1)
    assert w.U0.shape == (4, 256, 256) and w.U0.dtype == np.float64
    assert (w.steps, w.cfl, w.bc) == (200, 0.5, (0, 0, 0, 0))
    rho, u, v, p = _prim(w.U0)
    # four constant quadrants split at (0.5, 0.5), SW, SE, NW, NE in draw order
    quads = [rho[:128, :128], rho[128:, :128], rho[:128, 128:], rho[128:, 128:]]
    for k, (q, d) in enumerate(zip(quads, w.meta["quadrants"])):
        assert np.all(q == q.flat[0]), k
        r0, u0, v0, p0 = d
        assert 0.2 <= r0 <= 2 and -1 <= u0 <= 1 and -1 <= v0 <= 1 and 0.1 <= p0 <= 2
        assert math.isclose(q.flat[0], r0, rel_tol=0, abs_tol=0)
    assert np.allclose(p[:128, :128], w.meta["quadrants"][0][3], rtol=1e-12)
    # the seed decides the draws
    assert np.array_equal(workloads.riemann_quadrants(64, 64, seed=1).meta["quadrants"],
                          workloads.riemann_quadrants(32, 48, seed=1).meta["quadrants"])
    assert workloads.riemann_quadrants(64, 64, seed=2).meta["quadrants"] != w.meta["quadrants"]


def test_smooth_advection_is_exact_cell_averages(workloads):
    n = 64
    w = workloads.smooth_advection(n)
    assert (w.cfl, w.t_end, w.bc) == (0.4, 0.5, (2, 2, 2, 2))
    rho, u, v, p = _prim(w.U0)
    assert np.allclose(u, 1.0, rtol=1e-14) and np.allclose(v, 1.0, rtol=1e-14)
    assert np.allclose(p, 1.0, rtol=1e-13)
    # the exact state at t = 0.5 is the initial one (x + y moves by 1, the
    # period); at t = 1/n, x + y moves by two cells: a shift of 1 in x and 1 in y
    assert np.allclose(workloads.smooth_advection_exact(n, 0.5), rho, rtol=0, atol=1e-13)
    moved = workloads.smooth_advection_exact(n, 1.0 / n)
    assert np.allclose(moved, np.roll(np.roll(rho, 1, axis=0), 1, axis=1), rtol=0, atol=1e-13)
    # cell averages of sin over an h x h cell: the centre value times sinc^2
    h = 1.0 / n
    s = (math.sin(math.pi * h) / (math.pi * h)) ** 2
    assert w.meta["sinc2"] == s
    x = (np.arange(n) + 0.5) * h
    assert np.allclose(rho, 1.0 + 0.2 * s * np.sin(2 * np.pi * (x[:, None] + x[None, :])), rtol=0, atol=1e-15)


def test_mach3_cylinder(workloads):
    w = workloads.mach3_cylinder(2048, 1024)
    assert (w.nx, w.ny, w.lx, w.ly) == (2048, 1024, 2.0, 1.0)
    assert w.circle == (0.05, 0.4, 0.5) and w.steps == 3000 and w.cfl == 0.5
    rho, u, v, p = _prim(w.U0)
    assert np.all(rho == 1.4) and np.allclose(u, 3.0) and np.all(v == 0.0) and np.allclose(p, 1.0)
    assert math.isclose(3.0 / math.sqrt(GAMMA * 1.0 / 1.4), 3.0)     # Mach 3
    assert w.bc[0] == 1 and w.bc_prim[0] == [1.4, 3.0, 0.0, 1.0]     # Dirichlet inflow on the left


def test_shear_layer(workloads):
    n = 128
    w = workloads.shear_layer(n, seed=1)
    assert w.steps == 5000 and w.bc == (2, 2, 2, 2)
    assert math.isclose(w.meta["mu"], 1 / 2000) and w.meta["prandtl"] == 0.72
    a = np.array(w.meta["a"])
    assert a.shape == (8,) and np.all(np.abs(a) <= 1)
    rho, u, v, p = _prim(w.U0)
    assert np.allclose(rho, 1.0) and np.allclose(p, 2.5, rtol=1e-12)
    y = (np.arange(n) + 0.5) / n
    assert np.allclose(u[0], np.tanh((np.abs(y - 0.5) - 0.25) / 0.02) * np.where(y >= 0.5, 1, -1), atol=1e-14)
    x = (np.arange(n) + 0.5) / n
    vx = 0.01 * sum(a[k] * np.sin(2 * np.pi * (k + 1) * x) for k in range(8))
    assert np.allclose(v[:, 0], vx, atol=1e-15)


def test_uneven_batch(workloads):
    cases, states = workloads.batch_cases(512, seed=1)
    assert len(cases) == len(states) == 512
    sizes = np.array([(c["nx"], c["ny"]) for c in cases])
    assert sizes.min() >= 64 and sizes.max() <= 768 and np.all(sizes % 16 == 0)
    quads, cyls = cases[:256], cases[256:]
    assert all("circle" not in c for c in quads) and all("circle" in c for c in cyls)
    for c, U in zip(cyls, states[256:]):
        r, cx, cy = c["circle"]
        assert 0.03 <= r <= 0.1 and 3 * r <= cx <= 1 - 3 * r and 3 * r <= cy <= 1 - 3 * r
        rho, u, v, p = _prim(U[:, :1, :1])
        mach = u.item() / math.sqrt(GAMMA * p.item() / rho.item())
        assert 2.0 <= mach <= 3.0
    # the cells the bench reports for the batch
    assert int((sizes[:, 0] * sizes[:, 1]).sum()) == 90952704
