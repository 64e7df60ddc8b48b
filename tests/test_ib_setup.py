"""The engine's host immersed-boundary set-up (cfs_circle_setup in libcfs.so)
reproduces the reference's cell classification, immersed-ghost list, image
points and donor quadruples bit for bit (Circle.cpp:12-215)."""
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

GOLD = Path(__file__).resolve().parent / "golden"
has_ref = ob.REF_STRICT.exists() or ob.REFERENCE_TREE is not None


def test_cylinder_full_size_matches_reference_fixture(cfsb):
    g = dict(np.load(GOLD / "cylinder_2048x1024_lists.npz"))
    nx, ny, lx, ly = (int(g["grid"][0]), int(g["grid"][1]), float(g["grid"][2]), float(g["grid"][3]))
    r, cx, cy = g["circle"]
    types, cells, donors, images, normals = cfsb.circle_setup(nx, ny, lx, ly, r, cx, cy, 400)
    assert np.array_equal(np.flatnonzero(types.ravel() == 1), g["solid"])
    assert np.array_equal(cells, g["cells"])
    assert np.array_equal(donors, g["donors"])
    assert np.array_equal(images, g["images"])
    assert np.all(g["n_donors"] == 4)
    assert np.allclose(np.hypot(normals[:, 0], normals[:, 1]), 1.0, rtol=1e-14)


def test_cylinder_full_size_is_mirror_symmetric(cfsb):
    """The Mach-3 cylinder grid (2048 x 1024 on [0,2]x[0,1], body centred on
    y = 1/2): cell types are mirror images about that line exactly, every
    immersed ghost's mirror is a ghost whose donors are the mirrored donors,
    and the image points mirror to round-off (the polygon's vertices come from
    sin and cos, so they mirror to about one ulp; a normal is the unit vector
    from a ghost to its image point, whose length can be far below a cell, so
    its mirror error is that ulp over the length).  The FP64 flow's own mirror
    symmetry (tests/test_gpu_full_size.py) rests on this."""
    nx, ny = 2048, 1024
    types, cells, donors, images, normals = cfsb.circle_setup(nx, ny, 2.0, 1.0, 0.05, 0.4, 0.5, 400)
    assert np.array_equal(types, types[:, ::-1])
    i, j = cells // ny, cells % ny
    pos = {int(c): k for k, c in enumerate(cells)}
    mk = np.array([pos[int(c)] for c in i * ny + (ny - 1 - j)])
    mirrored = (donors[mk] // ny) * ny + (ny - 1 - donors[mk] % ny)
    assert np.array_equal(np.sort(donors, axis=1), np.sort(mirrored, axis=1))
    assert np.abs(images[:, 0] - images[mk, 0]).max() <= 4e-15
    assert np.abs(images[:, 1] - (1.0 - images[mk, 1])).max() <= 4e-15
    assert np.abs(normals[:, 1] + normals[mk, 1]).max() <= 1e-10


def test_small_circle_matches_reference_fixture(cfsb):
    g = dict(np.load(GOLD / "circle_64x64_lists.npz"))
    r, cx, cy = g["circle"]
    types, cells, donors, images, _ = cfsb.circle_setup(64, 64, 1.0, 1.0, r, cx, cy, 400)
    assert np.array_equal(types, g["types"])
    assert np.array_equal(cells, g["cells"])
    assert np.array_equal(donors, g["donors"])
    assert np.array_equal(images, g["images"])


@pytest.mark.skipif(not has_ref, reason="reference library not built here")
@pytest.mark.parametrize("nx,ny,lx,ly,circle,npts", [
    (96, 48, 2.0, 1.0, (0.1, 0.4, 0.5), 400),
    (80, 80, 1.0, 1.0, (0.23, 0.51, 0.47), 64),
    (128, 64, 2.0, 1.0, (0.07, 1.2, 0.33), 400),
    (50, 70, 1.0, 1.4, (0.3, 0.5, 0.7), 17),
    (12, 12, 1.0, 1.0, (0.55, 0.5, 0.5), 400),
])
def test_circle_setup_matches_live_reference(cfsb, nx, ny, lx, ly, circle, npts):
    rt, rc, rd, ri, rn = ob.ref_ib_info(nx, ny, lx, ly, circle, npoints=npts)
    if np.any(rn < 4):
        with pytest.raises(cfsb.CfsError):
            cfsb.circle_setup(nx, ny, lx, ly, *circle, npts)
        return
    types, cells, donors, images, _ = cfsb.circle_setup(nx, ny, lx, ly, *circle, npts)
    assert np.array_equal(types, rt)
    assert np.array_equal(cells, rc)
    assert np.array_equal(donors, rd)
    assert np.array_equal(images, ri)


def test_circle_without_enough_donors_is_rejected(cfsb):
    # A circle covering all but the grid corners: the reference warns and keeps a
    # 3-cell donor list (Circle.cpp:205-209), then reads past it in
    # ImagePoint::InterpolatePhase; the engine refuses the set-up instead.
    with pytest.raises(cfsb.CfsError) as e:
        cfsb.circle_setup(16, 16, 1.0, 1.0, 0.6, 0.5, 0.5, 400)
    assert e.value.code == 1 and "fluid donors" in str(e.value)


def test_no_circle_cells_when_outside(cfsb):
    types, cells, *_ = cfsb.circle_setup(32, 32, 1.0, 1.0, 0.05, 5.0, 5.0, 400)
    assert types.sum() == 0 and cells.size == 0
