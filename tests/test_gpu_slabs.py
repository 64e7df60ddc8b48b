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


def _steps_slab_run(cfsb, U, nsteps, prec, cfl, split):
    """The device-ordered path (cfs_steps_*): per stage the interior part,
    the halo exchange, the edge part; per step the CFL maximum exported,
    maxed and imported on the device.  The exchange between the two contexts'
    streams is ordered by host waits here (one GPU, two streams); between
    ranks NCCL orders it on the device."""
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
        buf = [torch.empty(nb, dtype=torch.uint8, device="cuda:0") for _ in range(4)]
        cfl_buf = torch.zeros(2, dtype=torch.int64, device="cuda:0")

        def pack():
            A.halo_pack(1, buf[0].data_ptr())
            A.halo_pack(0, buf[1].data_ptr())
            B.halo_pack(0, buf[2].data_ptr())
            B.halo_pack(1, buf[3].data_ptr())
            A.synchronize()
            B.synchronize()

        def unpack():
            B.halo_unpack(0, buf[0].data_ptr())
            B.halo_unpack(1, buf[1].data_ptr())
            A.halo_unpack(1, buf[2].data_ptr())
            A.halo_unpack(0, buf[3].data_ptr())

        def cfl_max():
            A.cfl_export(cfl_buf[0:1].data_ptr())
            B.cfl_export(cfl_buf[1:2].data_ptr())
            A.synchronize()
            B.synchronize()
            m = cfl_buf.max().reshape(1)
            torch.cuda.synchronize()
            A.cfl_import(m.data_ptr())
            B.cfl_import(m.data_ptr())
            A.synchronize()
            B.synchronize()

        pack()
        unpack()
        A.steps_begin(cfl=cfl)
        B.steps_begin(cfl=cfl)
        cfl_max()
        fresh = True
        for _ in range(nsteps):
            for _k in range(3):
                if not fresh:
                    pack()
                if split:
                    A.steps_stage(cfsb.PART_INTERIOR)
                    B.steps_stage(cfsb.PART_INTERIOR)
                if not fresh:
                    unpack()
                part = cfsb.PART_EDGES if split else cfsb.PART_ALL
                A.steps_stage(part)
                B.steps_stage(part)
                fresh = False
            cfl_max()
        ta, _ = A.steps_end()
        tb, _ = B.steps_end()
        assert ta == tb
        return np.concatenate([A.get_state(), B.get_state()], axis=1), ta
    finally:
        A.close()
        B.close()


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_device_ordered_slabs_equal_one_grid_advance(cfsb, workloads, prec, split):
    """Two slabs through cfs_steps_* (whole stages, or interior then edge rows)
    take the single grid's cfs_advance steps: the same dt sequence (the MAX of
    the slabs' fused CFL maxima is the grid's), FP64 bit for bit."""
    w = workloads.riemann_quadrants(96, 64, seed=11)
    got, t = _steps_slab_run(cfsb, w.U0, 5, prec, 0.45, split)
    with cfsb.Solver(96, 64, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                     bc=(cfsb.BC_PERIODIC,) * 4) as s:
        s.set_state(w.U0)
        tref, _ = s.advance(5, cfl=0.45)
        ref = s.get_state()
    if prec == 0:
        assert t == tref
        assert np.array_equal(got, ref)
    else:
        assert abs(t - tref) <= 1e-6 * tref
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_steps_api_state_errors(cfsb, workloads):
    w = workloads.riemann_quadrants(32, 32, seed=1)
    with cfsb.Solver(32, 32, precision=cfsb.FP64, bc=(cfsb.BC_PERIODIC,) * 4, rk=cfsb.RK_SSP3) as s:
        s.set_state(w.U0)
        with pytest.raises(cfsb.CfsError) as e:
            s.steps_stage(cfsb.PART_ALL)
        assert e.value.code == 4
        s.steps_begin(cfl=0.5)
        with pytest.raises(cfsb.CfsError) as e:
            s.steps_stage(cfsb.PART_EDGES)           # edges before the interior part
        assert e.value.code == 4
        s.steps_stage(cfsb.PART_INTERIOR)
        with pytest.raises(cfsb.CfsError) as e:
            s.steps_stage(cfsb.PART_ALL)             # the interior part awaits its edges
        assert e.value.code == 4
        s.steps_stage(cfsb.PART_EDGES)
        with pytest.raises(cfsb.CfsError) as e:
            s.steps_end()                            # inside a step
        assert e.value.code == 4
        s.steps_stage()
        s.steps_stage()
        t, dt = s.steps_end()
        assert t == dt > 0
