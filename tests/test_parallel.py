"""Slab decomposition (parallel.py) on CPU ranks over gloo: each rank advances
its slab with the C oracle on an extended array (its rows plus 3 ghost rows
per side), exchanging halos with parallel.HaloExchange after every stage and
taking the global CFL minimum; the assembled result must equal a single-domain
oracle run bit for bit."""
import ctypes
import importlib
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = "2d_compressible_flow_solver_b200"


def test_slab_bounds_and_neighbours():
    par = importlib.import_module(f"{PKG}.parallel")
    for nx, world in [(40, 2), (41, 3), (4096, 8), (7, 7)]:
        spans = [par.slab_bounds(nx, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == nx
        assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
        assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
    assert par.neighbours(1, 0, True) == (None, None)
    assert par.neighbours(2, 0, True) == (1, 1)
    assert par.neighbours(3, 0, False) == (None, 1)
    assert par.neighbours(3, 2, False) == (1, None)
    assert par.neighbours(4, 3, True) == (2, 0)


class OracleSlab:
    """HaloExchange adapter around the C oracle on an extended slab array."""

    def __init__(self, ob, U_slab, ny, dx, dy, bc_y, rk):
        self.ob = ob
        self.n = U_slab.shape[1]
        self.ny = ny
        self.cfg = ob.make_orc_config(self.n + 6, ny, lx=dx * (self.n + 6), ly=dy * ny, rk=rk, hll=1,
                                      bc=(0, 0, bc_y, bc_y))
        self.cfg_int = ob.make_orc_config(self.n, ny, lx=dx * self.n, ly=dy * ny, rk=rk, hll=1,
                                          bc=(0, 0, bc_y, bc_y))
        self.U = np.zeros((4, self.n + 6, ny))
        self.U[:, 3:3 + self.n] = U_slab
        self.U0 = np.zeros_like(self.U)
        self.U1 = np.zeros_like(self.U)
        self.rk = rk

    def nbytes(self):
        return 4 * 3 * self.ny * 8

    def _view(self, t):
        return t.numpy().view(np.float64).reshape(4, 3, self.ny)

    def pack(self, side, t):
        rows = slice(3, 6) if side == 0 else slice(self.n, self.n + 3)
        self._view(t)[:] = self.U[:, rows]

    def unpack(self, side, t):
        rows = slice(0, 3) if side == 0 else slice(self.n + 3, self.n + 6)
        self.U[:, rows] = self._view(t)

    def sync(self):
        pass

    def interior(self):
        return self.U[:, 3:3 + self.n].copy()

    def local_dt(self, cfl):
        return self.ob.orc_cfl_dt(self.cfg_int, np.ascontiguousarray(self.interior()), cfl)

    def stage(self, counter, dt):
        self.ob.orc_stage(self.cfg, self.U, self.U0, self.U1, self.ob.stage_of(self.rk, counter), dt)


def _worker(rank, world, port, U_global, steps, q):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import oracle_bind as ob

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        par = importlib.import_module(f"{PKG}.parallel")
        nx, ny = U_global.shape[1], U_global.shape[2]
        i0, i1 = par.slab_bounds(nx, world, rank)
        left, right = par.neighbours(world, rank, True)
        slab = OracleSlab(ob, U_global[:, i0:i1], ny, 1.0 / nx, 1.0 / ny, 2, ob.RK_SSP3)
        halo = par.HaloExchange(slab, dist, left, right, "cpu")
        halo.exchange()
        dts = []
        for _ in range(steps):
            dt = par.global_min(dist, slab.local_dt(0.45), "cpu")
            dts.append(dt)
            for k in range(1, 4):
                slab.stage(k, dt)
                halo.exchange()
        q.put((rank, i0, i1, slab.interior(), dts))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3, 4])
def test_slab_exchange_matches_single_domain(workloads, world):
    import oracle_bind as ob

    nx, ny, steps = 36, 20, 4
    U = workloads.riemann_quadrants(nx, ny, seed=8).U0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, U, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.zeros_like(U)
    for rank, i0, i1, part, dts in results:
        got[:, i0:i1] = part
    cfg = ob.make_orc_config(nx, ny, rk=ob.RK_SSP3, hll=1, bc=(2, 2, 2, 2))
    ref, ref_dt = ob.orc_run(cfg, U, 1, 3 * steps, cfl=0.45)
    assert np.array_equal(np.array(results[0][4]), ref_dt[::3])
    assert np.array_equal(got, ref)
