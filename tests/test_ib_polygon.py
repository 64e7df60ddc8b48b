"""Polygon immersed bodies (cfs_polygon_setup; no counterpart in the
reference, whose only shape is the circle), on the CPU: solid cells are the
centres inside the polygon, ghost cells follow the reference's marking walk,
each image point mirrors its ghost centre in the nearest boundary point and lies
outside the body, donors are fluid cells, and bad polygons are refused."""
import numpy as np
import pytest

from test_ib_marking_rule import order_free_ghosts


def _inside(xy, px, py):
    """Even-odd rule for many points."""
    inside = np.zeros(np.shape(px), dtype=bool)
    n = len(xy)
    for k in range(n):
        xk, yk = xy[k]
        xm, ym = xy[k - 1]
        cross = (yk > py) != (ym > py)
        with np.errstate(divide="ignore", invalid="ignore"):
            xint = (xm - xk) * (py - yk) / (ym - yk) + xk
        inside ^= cross & (px < xint)
    return inside


def _nearest_boundary(xy, p):
    best, q = np.inf, None
    for k in range(len(xy)):
        a, b = np.asarray(xy[k]), np.asarray(xy[(k + 1) % len(xy)])
        ab = b - a
        u = np.clip(np.dot(p - a, ab) / np.dot(ab, ab), 0.0, 1.0)
        c = a + u * ab
        d = np.linalg.norm(c - p)
        if d < best:
            best, q = d, c
    return best, q


SHAPES = {
    "square": [(0.4, 0.4), (0.6, 0.4), (0.6, 0.6), (0.4, 0.6)],
    "triangle": [(0.3, 0.35), (0.7, 0.5), (0.3, 0.65)],
    "l_shape": [(0.3, 0.3), (0.7, 0.3), (0.7, 0.45), (0.45, 0.45), (0.45, 0.7), (0.3, 0.7)],
}


@pytest.mark.parametrize("name", list(SHAPES))
def test_polygon_setup(cfsb, name):
    xy = SHAPES[name]
    nx, ny = 96, 80
    types, cells, donors, images, normals = cfsb.polygon_setup(nx, ny, 1.0, 1.0, xy)
    dx, dy = 1.0 / nx, 1.0 / ny
    X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dy, indexing="ij")
    solid = _inside(xy, X, Y)
    assert np.array_equal(types != 0, solid)
    assert np.array_equal(types == 2, order_free_ghosts(solid))
    assert np.array_equal(np.sort(cells), np.flatnonzero(types.ravel() == 2))
    assert np.all(types.ravel()[donors.ravel()] == 0)
    assert np.allclose(np.linalg.norm(normals, axis=1), 1.0)
    for g, c in enumerate(cells):
        p = np.array([(c // ny + 0.5) * dx, (c % ny + 0.5) * dy])
        d, q = _nearest_boundary(xy, p)
        assert np.allclose(images[g], p + 2 * (q - p), atol=1e-12)
        assert not _inside(xy, np.array(images[g][0]), np.array(images[g][1]))


def test_polygon_of_a_circle_matches_the_circle_up_to_its_chords(cfsb):
    nx = ny = 128
    r, cx, cy = 0.2, 0.5, 0.5
    k = np.arange(400)
    xy = np.stack([cx + r * np.cos(2 * np.pi * k / 400), cy + r * np.sin(2 * np.pi * k / 400)], axis=1)
    tp = cfsb.polygon_setup(nx, ny, 1.0, 1.0, xy)[0]
    tc = cfsb.circle_setup(nx, ny, 1.0, 1.0, r, cx, cy, 400)[0]
    X, Y = np.meshgrid((np.arange(nx) + 0.5) / nx, (np.arange(ny) + 0.5) / ny, indexing="ij")
    dist = np.hypot(X - cx, Y - cy)
    differ = (tp != 0) != (tc != 0)
    # only centres between a chord and the arc can differ
    assert np.all((dist[differ] > r * np.cos(np.pi / 400)) & (dist[differ] <= r))


def test_bad_polygons_are_refused(cfsb):
    with pytest.raises(cfsb.CfsError):
        cfsb.polygon_setup(32, 32, 1.0, 1.0, [(0.1, 0.1), (0.2, 0.2)])
    with pytest.raises(cfsb.CfsError):
        cfsb.polygon_setup(32, 32, 1.0, 1.0, [(0.1, 0.1), (np.nan, 0.2), (0.3, 0.1)])
