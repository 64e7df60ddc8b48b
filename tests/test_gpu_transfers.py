"""State transfers of large grids from and to pageable host arrays (the
chunked, threaded copies through a pinned staging buffer, csrc/host_stage.cpp)
move the same bytes as the plain copies of pinned arrays: the states are the
same bit for bit either way, in both throughput forms, for sizes whose byte
counts split unevenly over the chunks and threads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned_like(torch, a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    t.numpy()[:] = a
    return t


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nx,ny", [(2048, 2048), (1531, 1777)])
def test_pageable_and_pinned_transfers_agree(cfsb, workloads, prec, nx, ny):
    import torch

    assert 4 * nx * ny * 8 >= 32 << 20  # large enough for the staged copies
    rng = np.random.default_rng(nx + ny)
    w = workloads.riemann_quadrants(nx, ny, seed=3)
    U = w.U0 * (1.0 + 1e-3 * rng.standard_normal(w.U0.shape))
    U[3] += 1.0  # keep the pressure positive
    pin_in = _pinned_like(torch, U)
    pin_out = torch.empty(U.shape, dtype=torch.float64, pin_memory=True)
    kw = dict(precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4)
    with cfsb.Solver(nx, ny, **kw) as a, cfsb.Solver(nx, ny, **kw) as b:
        a.set_state(U)                 # pageable
        b.set_state(pin_in.numpy())    # pinned
        got_a = a.get_state()          # pageable
        b.get_state(pin_out.numpy())   # pinned
        assert np.array_equal(got_a, pin_out.numpy())
        if prec == cfsb.FP64:
            assert np.array_equal(got_a, U)
        a.advance(2, cfl=0.4)
        b.advance(2, cfl=0.4)
        after_a = a.get_state()
        b.get_state(pin_out.numpy())
        assert np.array_equal(after_a, pin_out.numpy())
        assert np.all(np.isfinite(after_a))
