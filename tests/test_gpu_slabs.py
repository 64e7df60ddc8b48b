"""Slab decomposition on one GPU, host-driven: two contexts with halo sides
(CFS_BC_HALO) exchange their 3 edge rows through cfs_halo_pack/unpack after
every stage (the messages parallel.HaloExchange sends between ranks) and take
the smaller CFL step.  The FP64 result must equal the single-grid run bit for
bit; FP32-mixed (shared storage offsets) to the form's rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _slab_run(cfsb, U, nsteps, prec, cfl):
    import torch

    nx, ny = U.shape[1], U.shape[2]
    h = nx // 2
    kw = dict(precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
              bc=(cfsb.BC_HALO, cfsb.BC_HALO, cfsb.BC_PERIODIC, cfsb.BC_PERIODIC))
    A = cfsb.Solver(h, ny, 0.5, 1.0, **kw)
    B = cfsb.Solver(nx - h, ny, (nx - h) / nx, 1.0, **kw)
    try:
        off = U.reshape(4, -1).mean(axis=1)
        for s, part in ((A, U[:, :h]), (B, U[:, h:])):
            s.set_storage_offsets(off)
            s.set_state(np.ascontiguousarray(part))
        nb = A.halo_bytes()
        assert nb == B.halo_bytes()
        buf = [torch.empty(nb, dtype=torch.uint8, device="cuda:0") for _ in range(4)]

        def exchange():
            # periodic in x: A's right edge -> B's left ghosts, B's right edge -> A's left ghosts, ...
            A.halo_pack(1, buf[0].data_ptr())
            A.halo_pack(0, buf[1].data_ptr())
            B.halo_pack(0, buf[2].data_ptr())
            B.halo_pack(1, buf[3].data_ptr())
            A.synchronize()
            B.synchronize()
            B.halo_unpack(0, buf[0].data_ptr())
            B.halo_unpack(1, buf[1].data_ptr())
            A.halo_unpack(1, buf[2].data_ptr())
            A.halo_unpack(0, buf[3].data_ptr())
            A.synchronize()
            B.synchronize()

        exchange()
        dts = []
        for _ in range(nsteps):
            dt = min(A.compute_dt(cfl), B.compute_dt(cfl))
            dts.append(dt)
            for k in (1, 2, 3):
                A.stage(k, dt)
                B.stage(k, dt)
                exchange()
        return np.concatenate([A.get_state(), B.get_state()], axis=1), dts
    finally:
        A.close()
        B.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_two_slabs_equal_one_grid(cfsb, workloads, prec):
    w = workloads.riemann_quadrants(96, 64, seed=11)
    U = w.U0
    got, dts = _slab_run(cfsb, U, 6, prec, 0.45)
    with cfsb.Solver(96, 64, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4) as s:
        s.set_state(U)
        for dt in dts:
            assert dt == s.compute_dt(0.45) or prec == 1
            s.step(dt)
        ref = s.get_state()
    if prec == 0:
        assert np.array_equal(got, ref)
    else:
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
