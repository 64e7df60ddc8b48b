"""Failure detection of the slab decomposition, injected on the host (CPU
ranks over gloo; no GPU is involved): a rank that dies between steps, with no
exchange or reduction in flight, makes its neighbour's next halo exchange or
CFL reduction fail with an error within the process group's timeout instead of
hanging; a rank that never joins makes the others' set-up fail the same way.
The engine's kernels never wait on another rank, so a failure can only surface
in these host-side collective steps."""
import importlib
import multiprocessing as mp
import os
import socket
import sys
import time
from datetime import timedelta
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = "2d_compressible_flow_solver_b200"


class _ArraySlab:
    """HaloExchange adapter over a plain array slab (3 ghost rows per side)."""

    def __init__(self, n, ny):
        self.U = np.zeros((4, n + 6, ny))
        self.n, self.ny = n, ny

    def nbytes(self):
        return 4 * 3 * self.ny * 8

    def _view(self, t):
        return t.numpy().view(np.float64).reshape(4, 3, self.ny)

    def pack(self, side, t):
        self._view(t)[:] = self.U[:, 3:6] if side == 0 else self.U[:, self.n:self.n + 3]

    def unpack(self, side, t):
        if side == 0:
            self.U[:, 0:3] = self._view(t)
        else:
            self.U[:, self.n + 3:self.n + 6] = self._view(t)

    def sync(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, die_after, q):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    par = importlib.import_module(f"{PKG}.parallel")
    t0 = time.monotonic()
    if die_after == -1 and rank == 1:
        os._exit(3)  # never joins
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    except Exception as e:
        q.put((rank, type(e).__name__, time.monotonic() - t0))
        q.close()
        q.join_thread()
        os._exit(0)
    slab = _ArraySlab(8, 16)
    left, right = par.neighbours(world, rank, True)
    halo = par.HaloExchange(slab, dist, left, right, "cpu")
    try:
        for step in range(6):
            if die_after is not None and rank == 1 and step == die_after:
                os._exit(3)  # dies between steps: nothing of it is in flight
            par.global_min(dist, 1.0 + rank, "cpu")
            for _ in range(3):
                halo.exchange()
        q.put((rank, "finished", time.monotonic() - t0))
    except Exception as e:  # the failure the survivor must see
        q.put((rank, type(e).__name__, time.monotonic() - t0))
        q.close()
        q.join_thread()  # the report is on its way before the process ends
        os._exit(0)
    dist.destroy_process_group()


def _run(world, die_after):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, die_after, q)) for r in range(world)]
    for p in procs:
        p.start()
    reports = {}
    deadline = time.monotonic() + 90
    expected = world if die_after is None else world - 1
    while len(reports) < expected and time.monotonic() < deadline:
        try:
            rank, what, secs = q.get(timeout=5)
            reports[rank] = (what, secs)
        except Exception:
            pass
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return reports, procs


def test_all_ranks_finish_without_a_fault():
    reports, procs = _run(2, None)
    assert all(reports[r][0] == "finished" for r in (0, 1)), reports
    assert all(p.exitcode == 0 for p in procs)


@pytest.mark.parametrize("world", [2, 3])
def test_a_rank_dying_between_steps_fails_its_neighbours_promptly(world):
    reports, procs = _run(world, die_after=2)
    survivors = [r for r in range(world) if r != 1]
    for r in survivors:
        assert r in reports, (r, reports)
        what, secs = reports[r]
        assert what != "finished", reports  # the exchange or the reduction raised
        assert secs < 60, reports            # within the group timeout, not a hang
    assert procs[1].exitcode == 3


def test_a_rank_that_never_joins_fails_the_set_up():
    reports, procs = _run(2, die_after=-1)
    assert 0 in reports, reports
    what, secs = reports[0]
    assert what != "finished" and secs < 60, reports
    assert procs[1].exitcode == 3
