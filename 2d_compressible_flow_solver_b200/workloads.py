"""Seeded synthetic workloads (initial states and settings) of the five
benchmark configurations.  The reference ships no datasets; its own initial
conditions are source/initialcondition/Reimman2D.cpp and Cylinder.cpp, and these
generators feed the engine through the same conserved-state interface
(``Initialcondition::fillIn``, Initialcondition.h:11).

Conserved energy is formed as EulerPhase::computeEnergyfromOther does
(EulerPhase.cpp:124-128): ``E = p/(gamma-1) + 0.5*(mx*mx + my*my)/rho`` with
``mx = rho*u``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GAMMA = 1.4


def conserved(rho, u, v, p, gamma: float = GAMMA) -> np.ndarray:
    rho = np.asarray(rho, dtype=np.float64)
    mx = rho * u
    my = rho * v
    E = p / (gamma - 1) + 0.5 * (mx * mx + my * my) / rho
    return np.stack(np.broadcast_arrays(rho, mx, my, E)).astype(np.float64)


def cell_centres(nx: int, ny: int, lx: float, ly: float):
    """Cell centres x = (i + 0.5) dx (CartesianMesh.cpp:92), shape (nx, ny)."""
    dx, dy = lx / nx, ly / ny
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    return np.meshgrid(x, y, indexing="ij")


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    lx: float
    ly: float
    U0: np.ndarray
    bc: tuple = (0, 0, 0, 0)
    bc_prim: list = field(default_factory=lambda: [[1.0, 0.0, 0.0, 1.0]] * 4)
    cfl: float = 0.5
    steps: int = 0
    t_end: float = 0.0
    circle: tuple | None = None          # (radius, cx, cy)
    meta: dict = field(default_factory=dict)


def riemann_quadrants(nx: int = 256, ny: int = 256, seed: int = 1) -> Workload:
    """Four-quadrant piecewise-constant state on [0,1]^2 split at (0.5, 0.5),
    quadrants drawn in the order SW, SE, NW, NE, each rho~U[0.2,2], u,v~U[-1,1],
    p~U[0.1,2]; transmissive (Neumann) sides as Reimman2D.cpp:41-51; CFL 0.5,
    200 steps."""
    rng = np.random.default_rng(seed)
    X, Y = cell_centres(nx, ny, 1.0, 1.0)
    rho = np.empty((nx, ny)); u = np.empty((nx, ny)); v = np.empty((nx, ny)); p = np.empty((nx, ny))
    quads = [(X < 0.5) & (Y < 0.5), (X >= 0.5) & (Y < 0.5), (X < 0.5) & (Y >= 0.5), (X >= 0.5) & (Y >= 0.5)]
    draws = []
    for m in quads:
        r0, u0, v0, p0 = rng.uniform(0.2, 2.0), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2.0)
        draws.append((r0, u0, v0, p0))
        rho[m], u[m], v[m], p[m] = r0, u0, v0, p0
    return Workload("riemann_quadrants", nx, ny, 1.0, 1.0, conserved(rho, u, v, p), cfl=0.5, steps=200,
                    meta={"seed": seed, "quadrants": draws})


def smooth_advection(n: int, t_end: float = 0.5) -> Workload:
    """rho = 1 + 0.2 sin(2 pi (x+y)), u = v = 1, p = 1, periodic [0,1]^2, CFL 0.4.
    Exact cell averages: the cell mean of sin(2 pi (x+y)) over an h x h cell is
    sin(2 pi (xc+yc)) (sin(pi h)/(pi h))^2, and every conserved variable is affine
    in rho, so the initial averages are exact.  The exact state at t is the
    initial one shifted by (t, t); at t = 0.5 it equals the initial state."""
    h = 1.0 / n
    X, Y = cell_centres(n, n, 1.0, 1.0)
    s = (math.sin(math.pi * h) / (math.pi * h)) ** 2
    rho = 1.0 + 0.2 * s * np.sin(2 * np.pi * (X + Y))
    U = np.stack([rho, rho, rho, 1.0 / (GAMMA - 1) + rho]).astype(np.float64)
    return Workload(f"smooth_advection_{n}", n, n, 1.0, 1.0, U, bc=(2, 2, 2, 2), cfl=0.4, t_end=t_end,
                    meta={"sinc2": s})


def smooth_advection_exact(n: int, t: float) -> np.ndarray:
    """Exact cell-averaged density of smooth_advection at time t."""
    h = 1.0 / n
    X, Y = cell_centres(n, n, 1.0, 1.0)
    s = (math.sin(math.pi * h) / (math.pi * h)) ** 2
    return 1.0 + 0.2 * s * np.sin(2 * np.pi * (X + Y - 2 * t))


def mach3_cylinder(nx: int = 2048, ny: int = 1024, radius: float = 0.05, cx: float = 0.4, cy: float = 0.5) -> Workload:
    """Mach-3 freestream (rho 1.4, u 3, v 0, p 1) on [0,2]x[0,1]: Dirichlet inflow
    on the left (Cylinder.cpp:22-32 style), Neumann elsewhere, circle of radius
    0.05 at (0.4, 0.5) with a 400-point polygon, 3000 steps at CFL 0.5."""
    prim = [1.4, 3.0, 0.0, 1.0]
    U = conserved(np.full((nx, ny), prim[0]), prim[1], prim[2], prim[3])
    return Workload("mach3_cylinder", nx, ny, 2.0, 1.0, U, bc=(1, 0, 0, 0), bc_prim=[prim] * 4, cfl=0.5,
                    steps=3000, circle=(radius, cx, cy))


def shear_layer(n: int = 1024, seed: int = 1, mu: float = 1.0 / 2000.0) -> Workload:
    """Periodic [0,1]^2 shear layer: rho 1, p 2.5,
    u = tanh((|y-0.5|-0.25)/0.02) sign(y-0.5) (sign(0) = 1),
    v = 0.01 sum_{k=1..8} a_k sin(2 pi k x) with a_k ~ U[-1,1]; mu = 1/2000
    (Re = 2000 with unit density, velocity and length), Pr 0.72, 5000 steps."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, size=8)
    X, Y = cell_centres(n, n, 1.0, 1.0)
    sgn = np.where(Y >= 0.5, 1.0, -1.0)
    u = np.tanh((np.abs(Y - 0.5) - 0.25) / 0.02) * sgn
    v = 0.01 * sum(a[k] * np.sin(2 * np.pi * (k + 1) * X) for k in range(8))
    U = conserved(np.ones((n, n)), u, v, 2.5)
    return Workload(f"shear_layer_{n}", n, n, 1.0, 1.0, U, bc=(2, 2, 2, 2), cfl=0.5, steps=5000,
                    meta={"seed": seed, "a": a.tolist(), "mu": mu, "prandtl": 0.72})


def batch_cases(ncases: int = 512, seed: int = 1, sizes=None):
    """Uneven batch: grid edges nx, ny drawn from {64, 80, ..., 768} (multiples of
    16); the first half are seeded four-quadrant states on [0,1]^2 with
    transmissive sides; the second half a Mach M ~ U[2, 3] freestream
    (rho 1.4, p 1, u = M sqrt(gamma p / rho)) past a circle of radius
    r ~ U[0.03, 0.1] centred in [3r, 1-3r]^2, Dirichlet inflow on the left,
    transmissive elsewhere, slip wall.  Every cell, those inside the body
    included, starts at the freestream: cells deeper in the body than the ghost
    layer keep that state and are still read by the fluid cells' 3-cell WENO
    stencils.  (The reference fills fluid cells only, Run.cpp:98-104, leaving
    zero-density solid cells inside those stencils.)  Returns (case
    descriptions, states)."""
    rng = np.random.default_rng(seed)
    edges = np.arange(64, 769, 16) if sizes is None else np.asarray(sizes)
    cases, states = [], []
    for k in range(ncases):
        nx, ny = int(rng.choice(edges)), int(rng.choice(edges))
        if k < ncases // 2:
            w = riemann_quadrants(nx, ny, seed=int(rng.integers(1 << 30)))
            cases.append({"nx": nx, "ny": ny, "lx": 1.0, "ly": 1.0, "bc": (0, 0, 0, 0)})
            states.append(w.U0)
        else:
            mach = rng.uniform(2.0, 3.0)
            r = rng.uniform(0.03, 0.1)
            cx, cy = rng.uniform(3 * r, 1 - 3 * r), rng.uniform(3 * r, 1 - 3 * r)
            rho, p = 1.4, 1.0
            u = mach * math.sqrt(GAMMA * p / rho)
            prim = [rho, u, 0.0, p]
            U = conserved(np.full((nx, ny), rho), u, 0.0, p)
            cases.append({"nx": nx, "ny": ny, "lx": 1.0, "ly": 1.0, "bc": (1, 0, 0, 0), "bc_prim": [prim] * 4,
                          "circle": (r, cx, cy), "ib_mode": 1})
            states.append(U)
    return cases, states

