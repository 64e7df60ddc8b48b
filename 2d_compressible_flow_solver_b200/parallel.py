"""Multi-GPU decomposition: one grid split into slabs along x, one slab per
rank (one GPU per rank), the B200 replacement of the reference's MPI
decomposition (source/parallel/CartesianParallel.cpp:3-60 decomposition,
:62-148 process-boundary ghost cells, :172-427 halo exchange).

Per RK stage each rank sends the 3 interior rows next to each inner side to
its neighbour and receives the neighbour's rows into its 3 ghost rows (rows
are contiguous in the engine's layout, so a message is 4 device copies of
3 x pitch elements).  Per step the CFL time step is the minimum over ranks.
Only the exchange is a collective step; everything else stays on each GPU.
The immersed boundary is not decomposed (a slab solver has none).  In the
FP32-mixed form every slab stores against the same offsets (the global means),
so the stored rows a message carries mean the same on both sides.

Message order (point-to-point ops match in posting order per peer): every
rank posts send(right rows -> right), send(left rows -> left),
recv(left ghost <- left), recv(right ghost <- right).  A rank's first message
to its right neighbour is therefore that neighbour's first receive from its
left, also when one rank is both neighbours (two ranks, periodic).

On the GPU nothing in a run of steps waits on the host (the engine's
cfs_steps_* entry points): the packs, the NCCL transfers, the unpacks and the
stage launches are ordered on the engine's stream (NCCL work joins it through
torch's stream semantics), the interior rows of each stage (which read no
ghost row) run while that stage's halo is in flight, the edge rows after it
lands, and the CFL step is the device-side maximum of every slab's fused CFL
maximum (one 8-byte MAX all-reduce per step on the same stream).  The
reference posts Irecv/Isend and waits on the host per stage
(CartesianParallel.cpp:285-295).
"""
from __future__ import annotations

import importlib
from pathlib import Path

_PKG = Path(__file__).resolve().parent.name


def slab_bounds(nx_global: int, world: int, rank: int) -> tuple[int, int]:
    """Rows [i0, i1) of `rank`: near-equal slabs, the first nx % world ranks one row longer."""
    base, extra = divmod(nx_global, world)
    i0 = rank * base + min(rank, extra)
    return i0, i0 + base + (1 if rank < extra else 0)


def neighbours(world: int, rank: int, periodic_x: bool) -> tuple[int | None, int | None]:
    """(left, right) ranks, None at a physical side of the global grid."""
    if world == 1:
        return None, None
    left = rank - 1 if rank > 0 else (world - 1 if periodic_x else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic_x else None)
    return left, right


class HaloExchange:
    """Ordered halo exchange of one slab.  `slab` provides nbytes(), pack(side,
    tensor), unpack(side, tensor) and sync(); `dist` is torch.distributed.
    `stream` (a torch stream, CUDA slabs): the stream the packs and unpacks are
    ordered on; the transfers are posted with it current, so NCCL waits for
    the packs on the device and the unpacks wait for NCCL on the device, with
    no host synchronisation.  Without a stream (CPU slabs) every call is
    synchronous."""

    def __init__(self, slab, dist, left, right, device, stream=None):
        import torch

        self.slab, self.dist, self.left, self.right = slab, dist, left, right
        self.stream = stream
        n = slab.nbytes()
        mk = lambda: torch.empty(n, dtype=torch.uint8, device=device)  # noqa: E731
        self.send = {0: mk(), 1: mk()}
        self.recv = {0: mk(), 1: mk()}

    def _ctx(self):
        import contextlib

        import torch

        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def start(self):
        """Packs the edge rows and posts the transfers; returns the requests."""
        if self.left is None and self.right is None:
            return []
        for side, peer in ((0, self.left), (1, self.right)):
            if peer is not None:
                self.slab.pack(side, self.send[side])
        if self.stream is None:
            self.slab.sync()
        d = self.dist
        ops = []
        if self.right is not None:
            ops.append(d.P2POp(d.isend, self.send[1], self.right))
        if self.left is not None:
            ops.append(d.P2POp(d.isend, self.send[0], self.left))
        if self.left is not None:
            ops.append(d.P2POp(d.irecv, self.recv[0], self.left))
        if self.right is not None:
            ops.append(d.P2POp(d.irecv, self.recv[1], self.right))
        with self._ctx():
            return d.batch_isend_irecv(ops)

    def finish(self, reqs) -> None:
        """Completes the transfers (on the device for CUDA slabs) and unpacks
        the received rows into the ghost rows."""
        if self.left is None and self.right is None:
            return
        with self._ctx():
            for req in reqs:
                req.wait()
        for side, peer in ((0, self.left), (1, self.right)):
            if peer is not None:
                self.slab.unpack(side, self.recv[side])

    def exchange(self) -> None:
        self.finish(self.start())


class _EngineSlab:
    """HaloExchange adapter of the CUDA engine (cfs_halo_* entry points)."""

    def __init__(self, solver):
        self.s = solver

    def nbytes(self):
        return self.s.halo_bytes()

    def pack(self, side, t):
        self.s.halo_pack(side, t.data_ptr())

    def unpack(self, side, t):
        self.s.halo_unpack(side, t.data_ptr())

    def sync(self):
        self.s.synchronize()


def global_min(dist, value: float, device) -> float:
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item())


class SlabSolver:
    """Engine solver of one slab of a global nx_global x ny grid on [0,lx]x[0,ly].
    bc is the global (left, right, bottom, top); inner x sides become halo sides.
    overlap (default): each stage updates its interior rows while its halo is
    exchanged, then its edge rows."""

    def __init__(self, nx_global: int, ny: int, lx: float, ly: float, *, dist, rank: int, world: int, device: int,
                 bc=(2, 2, 2, 2), overlap: bool = True, **solver_kw):
        import torch

        cfsb = importlib.import_module(_PKG)
        self.cfsb = cfsb
        self.dist, self.rank, self.world, self.device = dist, rank, world, device
        self.i0, self.i1 = slab_bounds(nx_global, world, rank)
        periodic_x = bc[0] == cfsb.BC_PERIODIC
        self.left, self.right = neighbours(world, rank, periodic_x)
        local_bc = list(bc)
        if self.left is not None:
            local_bc[0] = cfsb.BC_HALO
        if self.right is not None:
            local_bc[1] = cfsb.BC_HALO
        nloc = self.i1 - self.i0
        self.solver = cfsb.Solver(nloc, ny, lx * nloc / nx_global, ly, bc=tuple(local_bc), device=device, **solver_kw)
        self.stages = 2 if self.solver.config.rk == cfsb.RK_TVD2 else 3
        self.stream = torch.cuda.ExternalStream(self.solver.stream, device=f"cuda:{device}")
        self.halo = HaloExchange(_EngineSlab(self.solver), dist, self.left, self.right, f"cuda:{device}",
                                 stream=self.stream)
        self.exchanging = self.left is not None or self.right is not None
        self.overlap = overlap and self.exchanging and nloc >= 6
        self._cfl_buf = torch.zeros(1, dtype=torch.int64, device=f"cuda:{device}")
        self._ghosts_fresh = False

    def set_state(self, U_local) -> None:
        """Local conserved state [4][i1-i0][ny].  Halo messages carry stored
        values, so every slab of an FP32-mixed grid stores against the global
        means (one all-reduce of the local sums)."""
        import numpy as np
        import torch

        U_local = np.ascontiguousarray(U_local, dtype=np.float64)
        if self.world > 1:
            sums = torch.tensor([*U_local.reshape(4, -1).sum(axis=1), float(U_local[0].size)], dtype=torch.float64,
                                device=f"cuda:{self.device}")
            self.dist.all_reduce(sums, op=self.dist.ReduceOp.SUM)
            s = sums.cpu().numpy()
            self.solver.set_storage_offsets(s[:4] / s[4])
        self.solver.set_state(U_local)
        self.halo.exchange()
        self.solver.synchronize()
        self._ghosts_fresh = True

    def get_state(self):
        return self.solver.get_state()

    def compute_dt(self, cfl: float) -> float:
        dt = self.solver.compute_dt(cfl)
        return global_min(self.dist, dt, f"cuda:{self.device}") if self.world > 1 else dt

    def _cfl_allreduce(self) -> None:
        """MAX over ranks of the CFL maximum the next step uses, on the
        engine's stream (FP64 bits of non-negative values order as integers)."""
        if self.world == 1:
            return
        import torch

        self.solver.cfl_export(self._cfl_buf.data_ptr())
        with torch.cuda.stream(self.stream):
            self.dist.all_reduce(self._cfl_buf, op=self.dist.ReduceOp.MAX)
        self.solver.cfl_import(self._cfl_buf.data_ptr())

    def _stage(self) -> None:
        cfsb = self.cfsb
        reqs = None
        if self.exchanging and not self._ghosts_fresh:
            reqs = self.halo.start()
        if reqs is not None and self.overlap:
            self.solver.steps_stage(cfsb.PART_INTERIOR)
            self.halo.finish(reqs)
            self.solver.steps_stage(cfsb.PART_EDGES)
        else:
            if reqs is not None:
                self.halo.finish(reqs)
            self.solver.steps_stage(cfsb.PART_ALL)
        self._ghosts_fresh = False

    def advance(self, nsteps: int, cfl: float = 0.0, dt: float = 0.0) -> float:
        """nsteps RK steps with the global CFL dt (cfl > 0) or a fixed dt;
        returns the simulated time advanced.  One host wait, at the end."""
        self.solver.steps_begin(cfl=cfl, dt=dt)
        if cfl > 0:
            self._cfl_allreduce()
        for _ in range(nsteps):
            for _k in range(self.stages):
                self._stage()
            if cfl > 0:
                self._cfl_allreduce()
        t, _ = self.solver.steps_end()
        return t

    def step(self, dt: float) -> None:
        self.advance(1, dt=dt)

    def close(self) -> None:
        self.solver.close()
