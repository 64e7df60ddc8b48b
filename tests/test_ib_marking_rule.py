"""The device set-up marks immersed ghosts with an order-free rule (a non-fluid
cell is a ghost when, walking from it against one axis direction, the first
fluid cell lies within 3 steps on the grid) instead of the reference's walk
from every fluid cell (Circle.cpp:53-103).  This checks, on the CPU, that the
rule restated in numpy gives exactly the host set-up's types, which are pinned
to the reference's own classes."""
import numpy as np
import pytest


def order_free_ghosts(solid):
    nx, ny = solid.shape
    fluid = ~solid
    ghost = np.zeros_like(solid)
    for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        reach = np.zeros_like(solid)
        blocked = np.zeros_like(solid)  # a step left the grid earlier on the walk
        for m in range(1, 4):
            shifted = np.zeros_like(solid)
            inside = np.zeros_like(solid)
            # cell (i, j) looks at (i - m di, j - m dj)
            i0, i1 = max(0, m * di), nx + min(0, m * di)
            j0, j1 = max(0, m * dj), ny + min(0, m * dj)
            shifted[i0:i1, j0:j1] = fluid[i0 - m * di:i1 - m * di, j0 - m * dj:j1 - m * dj]
            inside[i0:i1, j0:j1] = True
            hit = shifted & inside & ~blocked & ~reach
            reach |= hit
            blocked |= ~inside
        ghost |= reach
    return ghost & solid


@pytest.mark.parametrize("seed", range(6))
def test_order_free_rule_equals_the_reference_walk(cfsb, seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(40, 200)), int(rng.integers(40, 200))
    r = rng.uniform(0.05, 0.3)
    cx, cy = rng.uniform(0.0, 1.0), rng.uniform(0.0, 1.0)
    try:
        types = cfsb.circle_setup(nx, ny, 1.0, 1.0, r, cx, cy, 400)[0]
    except cfsb.CfsError:
        pytest.skip("too few fluid donors for this circle")
    solid = types != 0
    assert np.array_equal(order_free_ghosts(solid), types == 2)
