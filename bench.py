#!/usr/bin/env python
"""Throughput benchmark of the stage engine: Mcell-steps/s on the smooth
periodic advection workload (rho = 1 + 0.2 sin(2 pi (x+y)), u = v = 1, p = 1 on
[0,1]^2, CFL 0.4, SSP-RK3, WENO5 eps 1e-2, Davis HLL) at 4096^2 cells, the
bandwidth-roofline configuration.  A step is one full RK3 step (3 fused stage
launches) over every cell; inputs are resident in HBM when timing starts.

Arms:
  default            the engine: FP32-mixed form (headline ``value``), with the
                     FP64 form, the FP32-vs-FP64 accuracy check at t = 0.5 on a
                     1024^2 grid, the end-to-end number through the C ABI with
                     pinned host buffers, the roofline and a CPU baseline (the
                     reference's own classes, timed on the host cores).
  --impl reference   the reference's own CPU implementation (oracle/_ref, built
                     with the reference Makefile's optimisation flags) on all host
                     cores, on bounded samples of the same workload.
  --workload batch   the uneven 512-case batch (persistent batched engine, FP32
                     and FP64) against a loop of plain FP64 solvers.
  --workload report  FP32-vs-FP64 accuracy, drift and rates on the quadrant,
                     Mach-3 cylinder, Navier-Stokes shear-layer and batch
                     configurations, and the circle set-up on host and device.
  --workload modes   the row march's feature sets on one 2048^2 grid.

Multi-GPU (torchrun, one rank per GPU, NCCL): one periodic grid of
(4096 N) x 4096 cells on [0, N] x [0, 1] split into N slabs of 4096^2 along x
(weak scaling, parallel.SlabSolver): after every stage each rank sends its 3
edge rows to its two neighbours and receives their rows into its ghost rows,
and every step takes the global minimum CFL time step.  Timings are the max
over ranks.  The batch workload splits its cases round-robin over the ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
PKG = "2d_compressible_flow_solver_b200"
METRIC = "Mcell-steps/s FP32-mixed vs FP64 on 1 B200 at ρ L1 err ≤1e-5; % HBM roofline"
UNIT = "Mcell-steps/s"
FALLBACK_HBM_GBS = 6650.0
# Algorithmic DRAM bytes per cell-step of SSP-RK3: stage 1 reads and writes U,
# stages 2 and 3 read U_s and U^n and write U -> 32 state words.
WORDS_PER_CELL_STEP = 32
# DRAM traffic of one stage launch per cell (dram__bytes_read.sum +
# dram__bytes_write.sum, averaged over the 3 stage launches of a step) from an
# ncu capture of the tuned FP32 march kernel on this 4096^2 workload (one pass
# per launch, the three stage launches of one warm step).
MEASURED_TRAFFIC_BYTES_PER_CELL_LAUNCH = {"f32": 41.6, "f64": None}
# Floating-point operations the FP32-mixed march executes per cell-step (its
# three stage launches; packed FFMA2 = 4, FADD2/FMUL2/FFMA/DFMA = 2, others 1),
# from ncu's per-opcode instruction counts (sass__inst_executed_per_opcode) of
# the three stage launches of one step on a periodic 2048^2 run with 32-row
# work items, as at 4096^2, and stochastic rounding in every stage (the
# defaults).  Data-independent on smooth states.
MEASURED_FLOPS_PER_CELL_STEP = {"f32": {"fp32": 2814.1, "fp64": 3.8}}
# The reference's scheme as its own driver runs it (Run.cpp:41-48 with
# TVD3rdRK, RiemmanSolverHLL, transmissive sides, fixed dt): what the
# reference arm times, and the engine's like-for-like companion rate.
REF_SCHEME_DT = 1e-4


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples of the GPU's SM clock and throttle reasons while the timed
    region runs: read-only NVML queries every 2 ms from a thread (nvidia-smi
    every 200 ms where NVML is missing).  open() and close() bracket the timed
    region; stop() reports the samples taken inside it (all samples if none
    fell inside, with "window": false)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event (throttle) reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = None
        self.samples = []  # (time, sm MHz, max sm MHz, reason names)
        self.t = None
        self.stop_flag = threading.Event()
        self.window = [None, None]

    def _handle(self, nv):
        # the CUDA device's NVML handle, by UUID (CUDA and NVML may number devices differently)
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:  # noqa: BLE001
            return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._handle(nv)
            smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.nvml = (nv, h, smax, get_reasons)
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return
        except Exception:  # noqa: BLE001
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read_smi, daemon=True)
        self.t.start()

    def open(self):
        self.window[0] = time.perf_counter()

    def close(self):
        self.window[1] = time.perf_counter()

    def _poll_nvml(self):
        nv, h, smax, get_reasons = self.nvml
        while not self.stop_flag.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                bits = int(get_reasons(h))
                names = [n for n, b in self.REASON_BITS.items() if bits & b]
                self.samples.append((time.perf_counter(), sm, smax, names))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.002)

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) < 9:
                continue
            try:
                sm, smax = float(f[1]), float(f[2])
            except ValueError:
                continue
            self.samples.append((time.perf_counter(), sm, smax, [n for k, n in enumerate(names)
                                                                 if f[5 + k].lower() == "active"]))

    def stop(self):
        if self.nvml is None and self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.t.join(timeout=2)
        t0, t1 = self.window
        inside = [x for x in self.samples if t0 is not None and t1 is not None and t0 <= x[0] <= t1]
        use = inside or self.samples
        sm = [x[1] for x in use]
        reasons = sorted({n for x in use for n in x[3]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(x[2] for x in use) if use else None,
                "reasons": reasons, "samples": len(use), "window": bool(inside),
                "source": "nvml (2 ms)" if self.nvml is not None else "nvidia-smi (200 ms)"}


# -------------------------------------------------- CPU reference timing
def _ref_sample_worker(args):
    """One bounded sample of the reference's own classes (perf build): one RK3
    step (3 Run::solver iterations) of the smooth workload on an n x n grid with
    transmissive sides (the reference has no periodic sides).  Returns
    (cells, seconds of the stage loop)."""
    n, root = args
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import oracle_bind as ob
    wl = importlib.import_module(f"{PKG}.workloads")
    lib = ob.ref_lib(perf=True)
    w = wl.smooth_advection(n)
    c = ob.make_ref_config(n, n, integrator=3, dt=1e-4)
    U = np.ascontiguousarray(w.U0)
    secs = lib.ref_time_stages(ctypes.byref(c), ob.P(U), 3)
    return n * n, secs


def cpu_reference_rate(nproc: int, n: int, rounds: int, warm: int = 0):
    """Aggregate Mcell-steps/s of nproc concurrent reference processes, each on
    its own n x n sample (the MPI build's per-rank work without its halo
    exchange).  Returns (rate per round list, seconds per round list)."""
    ctx = mp.get_context("spawn")
    rates, walls = [], []
    with ctx.Pool(nproc) as pool:
        for r in range(warm + rounds):
            t0 = time.perf_counter()
            res = pool.map(_ref_sample_worker, [(n, ROOT)] * nproc)
            wall = time.perf_counter() - t0
            if r >= warm:
                rates.append(sum(cells / secs for cells, secs in res) / 1e6)
                walls.append(wall)
    return rates, walls


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------- engine arm
def engine_arm(args):
    import torch
    import torch.distributed as dist

    rank, world, local = env_rank()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    cfsb = importlib.import_module(PKG)
    wl = importlib.import_module(f"{PKG}.workloads")
    n, K, W = args.n, args.steps, args.warmup
    w = wl.smooth_advection(n)
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4, device=local)

    def barrier():
        if world > 1:
            dist.barrier()

    autotune = importlib.import_module(f"{PKG}.autotune")
    variants = {cfsb.FP32_MIXED: autotune.best_variant("f32", n * n), cfsb.FP64: autotune.best_variant("f64", n * n)}

    def timed_advance_slab(prec, steps, warm, window=None):
        par = importlib.import_module(f"{PKG}.parallel")
        s = par.SlabSolver(n * world, n, float(world), 1.0, dist=dist, rank=rank, world=world, device=local,
                           bc=(cfsb.BC_PERIODIC,) * 4, precision=prec, variant=variants[prec], rk=cfsb.RK_SSP3,
                           hll=cfsb.HLL_DAVIS)
        # the field is 1-periodic in x, so every slab of [0, N] x [0, 1] starts
        # from the single-domain state
        s.set_state(w.U0)
        stream = torch.cuda.ExternalStream(s.solver.stream, device=local)
        if warm:
            s.advance(warm, w.cfl)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        if window:
            window.open()
        e0.record(stream)
        t_sim = s.advance(steps, w.cfl)
        e1.record(stream)
        torch.cuda.synchronize()
        if window:
            window.close()
        barrier()
        ms = e0.elapsed_time(e1)
        totals = s.solver.totals()
        s.close()
        return ms, t_sim, None, totals

    def timed_advance(prec, steps, warm, scheme=None, window=None):
        if world > 1:
            return timed_advance_slab(prec, steps, warm, window)
        skw, adv = dict(kw), dict(cfl=w.cfl)
        if scheme == "reference":
            skw.update(rk=cfsb.RK_TVD3_REFERENCE, hll=cfsb.HLL_REFERENCE, bc=(cfsb.BC_NEUMANN,) * 4)
            adv = dict(dt=REF_SCHEME_DT)
        s = cfsb.Solver(n, n, precision=prec, variant=variants[prec], **skw)
        s.set_state(w.U0)
        stream = torch.cuda.ExternalStream(s.stream, device=local)
        if warm:
            s.advance(warm, **adv)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        if window:
            window.open()
        e0.record(stream)
        t_sim, dt_last = s.advance(steps, **adv)
        e1.record(stream)
        torch.cuda.synchronize()
        if window:
            window.close()
        barrier()
        ms = e0.elapsed_time(e1)
        totals = s.totals()
        s.close()
        return ms, t_sim, dt_last, totals

    sampler = ClockSampler(local)
    sampler.start()
    ms32, t32, dt32, _ = timed_advance(cfsb.FP32_MIXED, K, W, window=sampler)
    clocks = sampler.stop()
    ms64, _, _, _ = timed_advance(cfsb.FP64, K, W)
    # the multi-GPU slab path at one rank (device-ordered stage launches through
    # the steps API, no graph, no exchange partner), against the single grid
    ms_slab1 = timed_advance_slab(cfsb.FP32_MIXED, K, W)[0] if world == 1 else None
    if world > 1:
        t = torch.tensor([ms32, ms64], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms32, ms64 = float(t[0]), float(t[1])
    cells = n * n
    v32 = cells * K * world / (ms32 / 1e3) / 1e6
    v64 = cells * K * world / (ms64 / 1e3) / 1e6

    result = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        bytes32 = WORDS_PER_CELL_STEP * 4 * cells * K
        achieved = bytes32 / (ms32 / 1e3) / 1e9
        # single grid: 3 stage launches per step + the first step's CFL
        # reduction; slabs: per stage an interior and two edge launches
        launches = 3 * K + 1 if world == 1 else 9 * K + 1
        per_launch_ms = ms32 / launches
        trf = MEASURED_TRAFFIC_BYTES_PER_CELL_LAUNCH["f32"]
        fl = MEASURED_FLOPS_PER_CELL_STEP["f32"]
        fp_peak = cfsb.fp_peaks(local)
        fp_achieved = (fl["fp32"] + fl["fp64"]) * cells * K / (ms32 / 1e3) / 1e12
        result = {
            "metric": METRIC, "value": round(v32, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": round(ms32 / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"smooth periodic advection {n}x{n} (rho=1+0.2 sin 2pi(x+y), u=v=1, p=1), "
                                   "SSP-RK3, WENO5 eps 1e-2, Davis HLL, CFL 0.4 on-device dt",
                       "precision": "fp32-mixed (FP32 storage, stochastic rounding in every stage)", "grid": [n, n],
                       "cells_per_gpu": cells,
                       "kernel_variant": {"f32": variants[cfsb.FP32_MIXED], "f64": variants[cfsb.FP64]},
                       "parallelism": "single grid" if world == 1 else
                       f"{world} slabs of {n}x{n} along x, 3-row halo exchange per stage (NCCL send/recv on the "
                       "engine's stream, overlapping the stage's interior rows), device-side global CFL max per step",
                       "l2": "inputs larger than L2 (3 state buffers of "
                             f"{4 * 4 * cells / 1e6:.0f} MB each)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} hbm_gbs",
                         "traffic": None if trf is None else round(trf * cells),
                         "traffic_is": "DRAM bytes per stage launch (ncu dram__bytes_read.sum + "
                                       "dram__bytes_write.sum of the FP32 march kernel on this 4096^2 workload)",
                         "algorithmic_bytes_per_cell_step": WORDS_PER_CELL_STEP * 4,
                         "avg_stage_launch_ms": round(per_launch_ms, 4),
                         "fp_pipe": {"achieved": round(fp_achieved, 2), "unit": "TFLOP/s",
                                     "peak": round(fp_peak["fp32_ffma"], 2),
                                     "frac": round(fp_achieved / fp_peak["fp32_ffma"], 4),
                                     "peak_source": "measured in this run (cfs_fp_peaks: FP32 FFMA chains; "
                                                    f"packed FFMA2 {fp_peak['fp32_ffma2']:.1f}, "
                                                    f"FP64 DFMA {fp_peak['fp64_dfma']:.1f} TFLOP/s)",
                                     "flops_per_cell_step": round(fl["fp32"] + fl["fp64"], 1),
                                     "flops_source": "ncu per-opcode thread-instruction counts of the FP32 march "
                                                     "kernel (periodic 2048^2)"}},
            "fp64": {"value": round(v64, 1), "ms_per_step": round(ms64 / K, 4),
                     "roofline_frac": round(WORDS_PER_CELL_STEP * 8 * cells * K / (ms64 / 1e3) / 1e9 / peak, 4),
                     "fp32_over_fp64": round(v32 / v64, 3)},
            "clocks": clocks,
            "gpu_launches": launches,
        }
        if ms_slab1 is not None:
            v_slab1 = cells * K / (ms_slab1 / 1e3) / 1e6
            result["slab_solver_1rank"] = {
                "fp32": round(v_slab1, 1), "over_single_grid": round(v_slab1 / v32, 4),
                "how": "parallel.SlabSolver at world size 1 on the same grid: the stages launched one by one "
                       "through the device-ordered steps API (no CUDA graph), CUDA events on the engine's stream"}
    # like-for-like companion of the reference arm: the reference's own scheme
    # (TVD3rdRK as written, its HLL, transmissive sides, fixed dt) on the same
    # 4096^2 state, FP64 and FP32-mixed
    if world == 1 and rank == 0:
        msr64, _, _, _ = timed_advance(cfsb.FP64, K, W, scheme="reference")
        msr32, _, _, _ = timed_advance(cfsb.FP32_MIXED, K, W, scheme="reference")
        result["same_scheme_as_reference_arm"] = {
            "scheme": f"TVD3rdRK as written + reference HLL + WENO5 eps 1e-2, transmissive sides, fixed dt "
                      f"{REF_SCHEME_DT}, {n}x{n}, smooth advection state",
            "fp64": round(cells * K / (msr64 / 1e3) / 1e6, 1), "fp32_mixed": round(cells * K / (msr32 / 1e3) / 1e6, 1),
            "timing": "CUDA events on the engine's stream, K steps after W warm-up steps"}
    # accuracy of FP32-mixed against FP64 at t_end (fixed dt so both forms sit
    # on the same time levels), and conservation drift
    if rank == 0 and args.accuracy_n > 0:
        ne = args.accuracy_n
        we = wl.smooth_advection(ne)
        with cfsb.Solver(ne, ne, precision=cfsb.FP64, **kw) as s:
            s.set_state(we.U0)
            dt0 = s.compute_dt(we.cfl)
        nsteps = int(math.ceil(we.t_end / dt0))
        dt = we.t_end / nsteps
        states = {}
        for prec in (cfsb.FP64, cfsb.FP32_MIXED):
            with cfsb.Solver(ne, ne, precision=prec, **kw) as s:
                s.set_state(we.U0)
                m0 = s.totals()
                s.advance(nsteps, dt=dt)
                states[prec] = (s.get_state(), m0, s.totals())
        U64, U32 = states[cfsb.FP64][0], states[cfsb.FP32_MIXED][0]
        m0, m1 = states[cfsb.FP32_MIXED][1], states[cfsb.FP32_MIXED][2]
        exact = wl.smooth_advection_exact(ne, we.t_end)
        result["accuracy"] = {
            "grid": [ne, ne], "t_end": we.t_end, "steps": nsteps,
            "rho_L1_fp32_vs_fp64": float(np.abs(U32[0] - U64[0]).mean()),
            "rho_Linf_fp32_vs_fp64": float(np.abs(U32[0] - U64[0]).max()),
            "E_L1_fp32_vs_fp64": float(np.abs(U32[3] - U64[3]).mean()),
            "E_Linf_fp32_vs_fp64": float(np.abs(U32[3] - U64[3]).max()),
            "mass_drift": float(abs(m1[0] - m0[0]) / abs(m0[0])),
            "energy_drift": float(abs(m1[3] - m0[3]) / abs(m0[3])),
            "rho_L1_fp64_vs_exact": float(np.abs(U64[0] - exact).mean()),
        }
    # end to end through the C ABI with pinned host buffers: initial state up,
    # K steps each reading back its dt and time, final state down; at N GPUs
    # every rank does this for its slab through parallel.SlabSolver (halo
    # exchange and the global CFL step included), wall time maxed over ranks
    pin = torch.empty((4, n, n), dtype=torch.float64, pin_memory=True)
    pin.numpy()[:] = w.U0
    out = torch.empty((4, n, n), dtype=torch.float64, pin_memory=True)
    if world == 1:
        with cfsb.Solver(n, n, precision=cfsb.FP32_MIXED, variant=variants[cfsb.FP32_MIXED], **kw) as s:
            s.set_state(pin.numpy())
            s.advance(2, cfl=w.cfl)
            s.synchronize()
            t0 = time.perf_counter()
            s.set_state(pin.numpy())
            for _ in range(K):
                s.advance(1, cfl=w.cfl)
            s.get_state(out.numpy())
            wall = time.perf_counter() - t0
            # the same with pageable host arrays, as a C++ caller's std::vector
            # (the library stages large pageable copies through pinned memory)
            # (warm: the staging buffer is pinned once per context, and the
            # output array's pages are touched once)
            host_out = np.empty((4, n, n))
            s.set_state(w.U0)
            s.get_state(host_out)
            s.synchronize()
            t0 = time.perf_counter()
            s.set_state(w.U0)
            for _ in range(K):
                s.advance(1, cfl=w.cfl)
            s.get_state(host_out)
            wall_pageable = time.perf_counter() - t0
    else:
        par = importlib.import_module(f"{PKG}.parallel")
        s = par.SlabSolver(n * world, n, float(world), 1.0, dist=dist, rank=rank, world=world, device=local,
                           bc=(cfsb.BC_PERIODIC,) * 4, precision=cfsb.FP32_MIXED,
                           variant=variants[cfsb.FP32_MIXED], rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS)
        s.set_state(pin.numpy())
        s.advance(2, w.cfl)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        s.set_state(pin.numpy())
        for _ in range(K):
            s.advance(1, w.cfl)
        s.solver.get_state(out.numpy())
        wall_t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(wall_t, op=dist.ReduceOp.MAX)
        wall = float(wall_t.item())
        s.close()
    if rank == 0:
        state_bytes = 4 * cells * 8
        result["e2e"] = {"value": round(cells * world * K / wall / 1e6, 1), "unit": UNIT, "steps": K,
                         "h2d_bytes_per_step": int(state_bytes / K + 40),
                         "d2h_bytes_per_step": int(state_bytes / K + 48),
                         "how": "per GPU: cfs_set_state from pinned host, K x cfs_advance(1) with dt/t read back "
                                "(at N GPUs through parallel.SlabSolver: halo exchange and global CFL step), "
                                "cfs_get_state to pinned host; host wall clock, max over ranks.  One FP64 state "
                                "(537 MB) per GPU goes up and one comes down per run, so the rate depends on K "
                                "(the steps field)"}
        if world == 1:
            result["e2e_pageable"] = {
                "value": round(cells * K / wall_pageable / 1e6, 1), "unit": UNIT, "steps": K,
                "how": "as e2e, with pageable host arrays (numpy) in place of pinned ones: cfs_set_state and "
                       "cfs_get_state copy them in 16 chunks through a pinned staging buffer, host threads "
                       "moving each chunk while the DMA engine moves the one before (after) it"}
    # the uneven 512-case batch (persistent batched engine), bounded: K steps
    # per form, device-timed with CUDA events on the batch's stream
    if rank == 0 and world == 1 and args.batch_cases > 0:
        result["batch"] = batch_subresult(cfsb, wl, torch, args.batch_cases, K, W, local)
    # CPU baseline: the reference's own classes on the host cores (rank 0, N=1)
    if rank == 0:
        if world == 1 and args.cpu_sample > 0:
            cores = host_cores()
            try:
                rates, walls = cpu_reference_rate(cores, args.cpu_sample, 1)
                result["cpu_baseline"] = {
                    "value": round(rates[0], 4), "unit": UNIT, "cores": cores, "kind": "reference",
                    "sample": f"{cores} concurrent single-rank processes of the reference's classes "
                              f"(-O3 -ffast-math build), each one RK3 step on a {args.cpu_sample}^2 grid of the "
                              f"same workload (transmissive sides); {walls[0]:.1f} s wall",
                }
            except Exception as e:  # noqa: BLE001
                result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                          "sample": f"unavailable: {e}"}
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ batch arm
def _time_batch(cfsb, torch, cases, states, prec, K: int, W: int, device: int):
    """(ms for K steps after W warm-up steps, cells, work items per stage) of
    one persistent batch, timed with CUDA events on the batch's stream (the
    per-case CFL reductions, graph replays and the final read-back of the
    per-case times included)."""
    with cfsb.Batch(cases, precision=prec, positivity=cfsb.POSITIVITY_FLOOR, device=device) as b:
        cells, items = b.info()
        for k, U in enumerate(states):
            b.set_state(k, U)
        b.advance(W, cfl=0.5)
        stream = torch.cuda.ExternalStream(b.stream, device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.advance(K, cfl=0.5)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), cells, items


def batch_subresult(cfsb, wl, torch, ncases: int, K: int, W: int, device: int) -> dict:
    """The uneven batch in the default line: every case of `ncases` (seeded,
    nx, ny in 64..768) advanced K steps after W warm-up steps by the persistent
    batched engine, FP32-mixed and FP64."""
    cases, states = wl.batch_cases(ncases, seed=1)
    out = {"workload": f"{ncases} uneven cases, nx,ny in 64..768 step 16, half four-quadrant, half Mach 2-3 "
                       "cylinder (slip wall), SSP-RK3, Davis HLL, positivity fallbacks with floors, per-case CFL 0.5",
           "steps": K, "warmup": W}
    for prec, key in ((cfsb.FP32_MIXED, "fp32"), (cfsb.FP64, "fp64")):
        ms, cells, items = _time_batch(cfsb, torch, cases, states, prec, K, W, device)
        out[key] = round(cells * K / (ms / 1e3) / 1e6, 1)
        out["cells"] = cells
        out["work_items_per_stage"] = items
    peak, kind = hbm_peak()
    out["value"] = out["fp32"]
    out["unit"] = UNIT
    out["fp32_over_fp64"] = round(out["fp32"] / out["fp64"], 3)
    out["hbm_frac_fp32"] = round(out["fp32"] * 1e6 * WORDS_PER_CELL_STEP * 4 / 1e9 / peak, 4)
    out["hbm_peak"] = f"{peak} GB/s ({kind})"
    return out


def batch_arm(args):
    """Uneven batch of independent cases (512 by default): aggregate
    Mcell-steps/s of the persistent batched engine (FP32-mixed and FP64) and of
    a loop of plain FP64 single-grid solvers over the same cases.  With N ranks
    each rank runs the cases k with k % N == rank; rates use the max wall time
    over ranks."""
    import torch
    import torch.distributed as dist

    rank, world, local = env_rank()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    cfsb = importlib.import_module(PKG)
    wl = importlib.import_module(f"{PKG}.workloads")
    cases, states = wl.batch_cases(args.cases, seed=1)
    cases, states = cases[rank::world], states[rank::world]
    K, W = args.steps, args.warmup

    def job_max(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def job_sum(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())
    out = {"workload": f"{args.cases} uneven cases, nx,ny in 64..768 step 16, half four-quadrant, half Mach 2-3 "
                       "cylinder (slip wall), SSP-RK3, Davis HLL, positivity fallbacks with floors, per-case CFL 0.5",
           "steps": K, "warmup": W}

    create_s = {}

    def run_batch(prec):
        t0 = time.perf_counter()
        with cfsb.Batch(cases, precision=prec, positivity=cfsb.POSITIVITY_FLOOR, device=local) as b:
            create_s[prec] = time.perf_counter() - t0
            cells, items = b.info()
            for k, U in enumerate(states):
                b.set_state(k, U)
            b.advance(W, cfl=0.5)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            b.advance(K, cfl=0.5)
            wall = job_max(time.perf_counter() - t0)
        cells = int(job_sum(cells))
        return cells, items, cells * K / wall / 1e6, wall

    cells, items, v32, w32 = run_batch(cfsb.FP32_MIXED)
    _, _, v64, w64 = run_batch(cfsb.FP64)
    out.update({"cells": cells, "work_items_per_stage": items,
                "batched_fp32": round(v32, 1), "batched_fp64": round(v64, 1),
                "create_s_fp32": round(create_s[cfsb.FP32_MIXED], 3)})
    # Per-case code paths: the same cases with the four-quadrant ones on
    # periodic sides, which need no edge code, so the batch runs two feature
    # groups (one persistent launch each per stage); against the same batch
    # with every case asking for the edge code (one group, one launch).
    periodic = [c if "circle" in c else dict(c, bc=(2, 2, 2, 2)) for c in cases]
    fg = {"workload": "the cases above with the four-quadrant cases on periodic sides (no edge code), "
                      "the cylinders unchanged; per-case code path (two launches per stage) against the edge "
                      "code for every case (cfs_case.edge_code = 1, one launch per stage); CUDA events on the "
                      "batch's stream, max over ranks"}
    for label, cs in (("per_case", periodic), ("edge_code_for_all", [dict(c, edge_code=True) for c in periodic])):
        for prec, key in ((cfsb.FP32_MIXED, "fp32"), (cfsb.FP64, "fp64")):
            ms, c_cells, _ = _time_batch(cfsb, torch, cs, states, prec, K, W, local)
            fg[f"{label}_{key}"] = round(job_sum(c_cells) * K / (job_max(ms) / 1e3) / 1e6, 1)
    fg["per_case_gain_fp32"] = round(fg["per_case_fp32"] / fg["edge_code_for_all_fp32"], 3)
    fg["per_case_gain_fp64"] = round(fg["per_case_fp64"] / fg["edge_code_for_all_fp64"], 3)
    out["feature_groups"] = fg
    solvers = []
    for c, U in zip(cases, states):
        s = cfsb.Solver(c["nx"], c["ny"], c["lx"], c["ly"], precision=cfsb.FP64, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                        bc=c["bc"], bc_prim=c.get("bc_prim"), positivity=cfsb.POSITIVITY_FLOOR, device=local)
        if "circle" in c:
            s.build_circle(*c["circle"], 400, cfsb.IB_BILINEAR_SLIP)
        s.set_state(U)
        s.advance(W, cfl=0.5)
        solvers.append(s)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for s in solvers:
        s.advance(K, cfl=0.5)
    wall = job_max(time.perf_counter() - t0)
    for s in solvers:
        s.close()
    loop64 = cells * K / wall / 1e6
    peak, _ = hbm_peak()
    out.update({"loop_plain_fp64": round(loop64, 1), "batched_fp32_over_loop_fp64": round(v32 / loop64, 2),
                "batched_fp32_over_batched_fp64": round(v32 / v64, 2),
                "batched_fp32_hbm_frac": round(v32 * 1e6 * WORDS_PER_CELL_STEP * 4 / 1e9 / peak, 4),
                "timing": "host wall clock around cfs_batch_advance / the per-case cfs_advance loop (each call "
                          "waits for its stream), max over ranks", "n_gpus": world})
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ report arm
def _errors(a, b):
    """L1 / L-infinity of rho and E between two states."""
    return {"rho_L1": float(np.abs(a[0] - b[0]).mean()), "rho_Linf": float(np.abs(a[0] - b[0]).max()),
            "E_L1": float(np.abs(a[3] - b[3]).mean()), "E_Linf": float(np.abs(a[3] - b[3]).max())}


def _perturbed(U, kind: str, seed: int = 7):
    """U with every value moved by a random-sign relative amount: one FP64 ulp
    ("ulp64") or the FP32 unit roundoff 2^-24 ("u32")."""
    rng = np.random.default_rng(seed)
    sign = rng.choice([-1.0, 1.0], size=U.shape)
    if kind == "ulp64":
        return np.where(sign > 0, np.nextafter(U, np.inf), np.nextafter(U, -np.inf))
    return U * (1.0 + sign * 2.0 ** -24)


def report_arm(args):
    """Accuracy and conservation of the FP32-mixed form against FP64, every
    comparison on ONE time-step sequence: the FP64 run takes its CFL steps one
    advance call at a time and records each dt; the other runs replay that
    sequence with fixed steps, so both forms end at the same t_end.
    Configurations: four-quadrant Riemann problems (256^2, 200 steps, the
    reference's scheme: TVD3 as written + its HLL; the FP64 form also against
    the exact form, the reference's arithmetic), the Mach-3 cylinder (2048 x
    1024, 3000 steps, slip wall, positivity fallbacks with floors), the
    Navier-Stokes shear layer (1024^2, 5000 steps) and the uneven batch (512
    cases, 500 steps).  Beside each FP32 error, the sensitivity of the FP64
    run itself: the difference at t_end made by perturbing its initial state
    by one FP64 ulp, and by the FP32 unit roundoff, per value (random signs).
    Then the smooth-advection convergence table (FP64 and FP32 against the
    exact solution at t = 0.5, N = 128 .. --conv-max).  Open boundaries:
    drift is the FP32-vs-FP64 difference of the totals; periodic: the change
    of each form's totals.  One JSON line."""
    import torch

    torch.cuda.set_device(0)
    cfsb = importlib.import_module(PKG)
    wl = importlib.import_module(f"{PKG}.workloads")
    out = {"report": "FP32-mixed vs FP64 at t_end on one time-step sequence per configuration"}

    def solver(w, prec, extra, circle=None, ib_mode=None):
        s = cfsb.Solver(w.nx, w.ny, w.lx, w.ly, precision=prec, bc=w.bc, bc_prim=w.bc_prim, **extra)
        if circle is not None:
            s.build_circle(*circle, 400, ib_mode)
        return s

    def run_cfl(w, prec, steps, cfl, extra, circle, ib_mode):
        with solver(w, prec, extra, circle, ib_mode) as s:
            s.set_state(w.U0)
            m0 = s.totals()
            dts = []
            t0 = time.perf_counter()
            for _ in range(steps):
                dts.append(s.advance(1, cfl=cfl)[1])
            wall = time.perf_counter() - t0
            return s.get_state(), m0, s.totals(), np.array(dts), wall

    def run_dts(w, prec, dts, extra, circle, ib_mode, U0=None):
        with solver(w, prec, extra, circle, ib_mode) as s:
            s.set_state(w.U0 if U0 is None else U0)
            m0 = s.totals()
            t0 = time.perf_counter()
            for dt in dts:
                s.advance(1, dt=float(dt))
            wall = time.perf_counter() - t0
            return s.get_state(), m0, s.totals(), wall

    def compare(name, w, steps, cfl, extra, circle=None, ib_mode=None, exact=False, periodic=False):
        U64, m0_64, m1_64, dts, wall64 = run_cfl(w, cfsb.FP64, steps, cfl, extra, circle, ib_mode)
        U32, m0_32, m1_32, wall32 = run_dts(w, cfsb.FP32_MIXED, dts, extra, circle, ib_mode)
        row = {"grid": [w.nx, w.ny], "steps": steps, "t_end": float(dts.sum()),
               "dt_sequence": "FP64 CFL steps, replayed as fixed steps by the other runs",
               "fp32_vs_fp64": _errors(U32, U64),
               "finite": bool(np.all(np.isfinite(U64)) and np.all(np.isfinite(U32))),
               "mcell_steps_per_s_one_step_per_call": {"fp64": round(w.nx * w.ny * steps / wall64 / 1e6, 1),
                                                       "fp32": round(w.nx * w.ny * steps / wall32 / 1e6, 1)}}
        sens = {}
        for kind in ("ulp64", "u32"):
            Up = _perturbed(w.U0, kind)
            Ux, _, _, _ = run_dts(w, cfsb.FP64, dts, extra, circle, ib_mode, U0=Up)
            d0 = float(np.abs(Up[0] - w.U0[0]).mean())
            e = _errors(Ux, U64)
            sens[kind] = {"rho_L1_initial": d0, "rho_L1_at_t_end": e["rho_L1"], "rho_Linf_at_t_end": e["rho_Linf"],
                          "amplification_L1": e["rho_L1"] / d0 if d0 > 0 else None}
        row["fp64_sensitivity"] = sens
        if periodic:
            row["drift_fp32"] = {"mass": float(abs(m1_32[0] - m0_32[0]) / abs(m0_32[0])),
                                 "energy": float(abs(m1_32[3] - m0_32[3]) / abs(m0_32[3]))}
            row["drift_fp64"] = {"mass": float(abs(m1_64[0] - m0_64[0]) / abs(m0_64[0])),
                                 "energy": float(abs(m1_64[3] - m0_64[3]) / abs(m0_64[3]))}
        else:
            row["totals_fp32_vs_fp64"] = {"mass": float(abs(m1_32[0] - m1_64[0]) / abs(m1_64[0])),
                                          "energy": float(abs(m1_32[3] - m1_64[3]) / abs(m1_64[3]))}
        if exact:
            Ue, _, _, _ = run_dts(w, cfsb.FP64_EXACT, dts, extra, circle, ib_mode)
            row["fp64_vs_exact_form"] = _errors(U64, Ue)
            row["exact_form_finite"] = bool(np.all(np.isfinite(Ue)))
        out[name] = row
        print(json.dumps({name: row}), file=sys.stderr, flush=True)

    parts = args.report_parts.split(",")
    if "quadrants" in parts:
        compare("quadrants_256_reference_scheme", wl.riemann_quadrants(256, 256, seed=1), 200, 0.5,
                dict(rk=cfsb.RK_TVD3_REFERENCE, hll=cfsb.HLL_REFERENCE), exact=True)
    if "cylinder" in parts:
        w3 = wl.mach3_cylinder(2048, 1024)
        compare("mach3_cylinder_2048x1024", w3, 3000, 0.5,
                dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, positivity=cfsb.POSITIVITY_FLOOR),
                circle=w3.circle, ib_mode=cfsb.IB_BILINEAR_SLIP)

        def best_s(fn, reps=3):
            best = None
            for _ in range(reps):
                t0 = time.perf_counter()
                r = fn()
                dt = time.perf_counter() - t0
                best = dt if best is None or dt < best else best
            return best, r
        geo = (w3.nx, w3.ny, w3.lx, w3.ly, *w3.circle, 400)
        th, rh = best_s(lambda: cfsb.circle_setup(*geo))
        td, rd = best_s(lambda: cfsb.circle_setup(*geo, device=0))
        out["ib_setup_2048x1024"] = {"host_ms": round(th * 1e3, 2), "device_ms": round(td * 1e3, 2),
                                     "ghost_cells": int(rh[1].size),
                                     "identical": all(np.array_equal(a, b) for a, b in zip(rh, rd)),
                                     "timing": "host wall clock, best of 3, both through the C ABI with host outputs"}
    if "shear" in parts:
        w4 = wl.shear_layer(1024)
        compare("shear_layer_1024_ns", w4, 5000, 0.5,
                dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, viscous=cfsb.VISCOUS_NS, mu=w4.meta["mu"], prandtl=0.72,
                     mach=1.0), periodic=True)
    if "batch" in parts:
        out[f"batch_{args.cases}_cases_{args.batch_steps}_steps"] = _report_batch(cfsb, wl, args.cases, args.batch_steps)
    if "convergence" in parts:
        out["convergence_smooth_advection"] = _report_convergence(cfsb, wl, args.conv_max)
    print(json.dumps(out), flush=True)


def _report_batch(cfsb, wl, ncases: int, steps: int) -> dict:
    """The uneven batch: FP64 with per-case CFL steps (one advance call per
    step, each case's dt recorded), FP32-mixed replaying every case's dt
    sequence; worst case over the cases at t_end."""
    cases, states = wl.batch_cases(ncases, seed=1)
    kw = dict(positivity=cfsb.POSITIVITY_FLOOR)
    with cfsb.Batch(cases, precision=cfsb.FP64, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        seq = []
        for _ in range(steps):
            b.advance(1, cfl=0.5)
            seq.append(b.dt_last())
        t64 = np.sum(seq, axis=0)
        U64 = [b.get_state(k) for k in range(len(cases))]
    with cfsb.Batch(cases, precision=cfsb.FP32_MIXED, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        t32 = np.zeros(len(cases))
        for d in seq:
            t32 += b.advance(1, dt=d)
        U32 = [b.get_state(k) for k in range(len(cases))]
    worst = {"rho_L1": 0.0, "rho_Linf": 0.0, "E_L1": 0.0, "E_Linf": 0.0}
    l1 = []
    finite = True
    for a, c in zip(U32, U64):
        e = _errors(a, c)
        l1.append(e["rho_L1"])
        finite = finite and bool(np.all(np.isfinite(a)) and np.all(np.isfinite(c)))
        for k in worst:
            worst[k] = max(worst[k], e[k])
    l1 = np.array(l1)
    half = len(cases) // 2
    return {"worst_case_fp32_vs_fp64": worst, "finite": finite, "steps": steps,
            "rho_L1_median": float(np.median(l1)),
            "rho_L1_worst_quadrant_case": float(l1[:half].max()), "rho_L1_worst_cylinder_case": float(l1[half:].max()),
            "cases_over_1e-5": int((l1 > 1e-5).sum()),
            "same_t_end": bool(np.allclose(t32, t64, rtol=1e-12, atol=0.0)),
            "dt_sequence": "per case: FP64 CFL steps, replayed by the FP32 batch (cfs_batch_advance_dt)"}


def _report_convergence(cfsb, wl, nmax: int) -> dict:
    """Smooth periodic advection to t = 0.5 at CFL <= 0.4 (fixed dt = 0.5 /
    ceil(0.5 / dt_CFL), so t_end is exact), SSP-RK3, Davis HLL, WENO5 eps 1e-2:
    density L1 error against the exact cell averages per N, FP64 and FP32, the
    observed order log2(e(N/2) / e(N)), and FP32 vs FP64."""
    rows = []
    kw = dict(rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4)
    n = 128
    prev = None
    while n <= nmax:
        w = wl.smooth_advection(n)
        with cfsb.Solver(n, n, precision=cfsb.FP64, **kw) as s:
            s.set_state(w.U0)
            dt0 = s.compute_dt(w.cfl)
        nsteps = int(math.ceil(w.t_end / dt0))
        dt = w.t_end / nsteps
        exact = wl.smooth_advection_exact(n, w.t_end)
        res = {}
        for prec, key, rnd in ((cfsb.FP64, "fp64", cfsb.ROUND_STOCHASTIC_ALL), (cfsb.FP32_MIXED, "fp32", cfsb.ROUND_STOCHASTIC_ALL),
                               (cfsb.FP32_MIXED, "fp32_sr_last", cfsb.ROUND_STOCHASTIC)):
            with cfsb.Solver(n, n, precision=prec, rounding=rnd, **kw) as s:
                s.set_state(w.U0)
                m0 = s.totals()
                s.advance(nsteps, dt=dt)
                U = s.get_state()
                m1 = s.totals()
            res[key] = (U, float(np.abs(U[0] - exact).mean()), float(abs(m1[0] - m0[0]) / abs(m0[0])))
        row = {"n": n, "steps": nsteps, "dt": dt,
               "rho_L1_fp64_vs_exact": res["fp64"][1], "rho_L1_fp32_vs_exact": res["fp32"][1],
               "rho_L1_fp32_vs_fp64": float(np.abs(res["fp32"][0][0] - res["fp64"][0][0]).mean()),
               "rho_Linf_fp32_vs_fp64": float(np.abs(res["fp32"][0][0] - res["fp64"][0][0]).max()),
               "mass_drift_fp64": res["fp64"][2], "mass_drift_fp32": res["fp32"][2],
               "rho_L1_fp32_sr_last_stage_vs_fp64": float(np.abs(res["fp32_sr_last"][0][0] - res["fp64"][0][0]).mean()),
               "mass_drift_fp32_sr_last_stage": res["fp32_sr_last"][2]}
        if prev is not None:
            row["order_fp64"] = math.log2(prev["rho_L1_fp64_vs_exact"] / row["rho_L1_fp64_vs_exact"])
            row["order_fp32"] = math.log2(prev["rho_L1_fp32_vs_exact"] / row["rho_L1_fp32_vs_exact"])
        rows.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
        prev = row
        n *= 2
    return {"rows": rows, "scheme": "SSP-RK3, Davis HLL, WENO5 eps 1e-2 (Weno5th.cpp:5), CFL <= 0.4, t = 0.5"}


# ----------------------------------------------------------- reference arm
# Bytes the reference's object graph holds per cell (Cell, faces, phases,
# fluxes, stencil lists), measured on its own build: about 2.2 KB; the arm sizes
# its tiles against the host's available memory with this figure.
REF_BYTES_PER_CELL = 2500


def _ref_tile_worker(conn, n: int, root: str) -> None:
    """One host core's share of the reference arm: builds an n x n grid of the
    smooth workload with the reference's own classes (perf build) once, then
    on each request runs one RK step (3 Run::solver iterations of TVD3rdRK) and
    returns the stage loop's wall-clock seconds."""
    sys.path.insert(0, root)
    sys.path.insert(0, str(Path(root) / "tests"))
    import oracle_bind as ob
    wl = importlib.import_module(f"{PKG}.workloads")
    lib = ob.ref_lib(perf=True)
    lib.ref_session_create.restype = ctypes.c_void_p
    lib.ref_session_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.ref_session_stages.restype = ctypes.c_double
    lib.ref_session_stages.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_session_destroy.restype = None
    lib.ref_session_destroy.argtypes = [ctypes.c_void_p]
    U = np.ascontiguousarray(wl.smooth_advection(n).U0)
    c = ob.make_ref_config(n, n, integrator=3, dt=REF_SCHEME_DT)
    t0 = time.perf_counter()
    h = lib.ref_session_create(ctypes.byref(c), ob.P(U))
    del U
    conn.send(("ready", time.perf_counter() - t0))
    while True:
        msg = conn.recv()
        if msg is None:
            break
        conn.send(lib.ref_session_stages(h, 3))
    lib.ref_session_destroy(h)
    conn.close()


def ref_tiles_rate(cores: int, n: int, steps: int, warm: int) -> dict:
    """`cores` concurrent reference processes, one n x n tile each: every step
    all of them run one RK step; the step's time is the host wall clock from the
    request to the last answer.  Returns the rate over the timed steps."""
    ctx = mp.get_context("spawn")
    procs, pipes = [], []
    for _ in range(cores):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_tile_worker, args=(b, n, str(ROOT)), daemon=True)
        pr.start()
        procs.append(pr)
        pipes.append(a)
    try:
        build = max(pp.recv()[1] for pp in pipes)
        walls = []
        for k in range(warm + steps):
            t0 = time.perf_counter()
            for pp in pipes:
                pp.send(1)
            for pp in pipes:
                pp.recv()
            if k >= warm:
                walls.append(time.perf_counter() - t0)
    finally:
        for pp in pipes:
            try:
                pp.send(None)
            except (BrokenPipeError, OSError):
                pass
        for pr in procs:
            pr.join(timeout=60)
    total = sum(walls)
    cells = cores * n * n
    return {"value": cells * steps / total / 1e6, "ms_per_step": total / steps * 1e3, "cells_per_step": cells,
            "build_s": build, "step_walls_s": [round(x, 3) for x in walls]}


def reference_arm(args):
    """The reference's own CPU implementation of the path (its classes built
    with its Makefile's optimisation flags, oracle/_ref/libref_perf.so) on all
    host cores: one single-rank process per core, each holding its own tile of
    the smooth workload, all stepping together (the MPI build's per-rank work
    without its halo exchange, CartesianParallel.cpp:3-47).  The tiles add up
    to the engine's n x n cells when the host's memory allows (about 2.2 KB per
    cell in the reference's object graph), else to the largest share it allows;
    the line reports the cells actually stepped and the measured time per step,
    nothing extrapolated."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    cores = host_cores()
    lib = ROOT / "oracle" / "_ref" / "libref_perf.so"
    if not lib.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_perf.so not built "
                          "(needs the reference tree; run __graft_entry__.build())"}), flush=True)
        return
    n = args.ref_tile
    if n <= 0:
        n = int(args.n / math.sqrt(cores)) // 16 * 16
        try:
            import psutil
            avail = psutil.virtual_memory().available
            while n > 64 and cores * n * n * REF_BYTES_PER_CELL > 0.6 * avail:
                n -= 64
        except ImportError:
            pass
    r = ref_tiles_rate(cores, n, args.steps, args.warmup)
    v = r["value"]
    workload = (f"smooth advection state (rho=1+0.2 sin 2pi(x+y), u=v=1, p=1) as {cores} independent {n}x{n} tiles "
                f"= {r['cells_per_step']} cells per step (engine line: {args.n}x{args.n} = {args.n * args.n}), "
                f"one single-rank reference process per host core; TVD3rdRK as written, reference HLL "
                f"(RiemmanSolverHLL), WENO5 eps 1e-2, transmissive sides, fixed dt {REF_SCHEME_DT}")
    out = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms_per_step"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "tiles": cores, "tile": [n, n], "cells_per_step": r["cells_per_step"],
                   "precision": "reference FP64 (its Makefile's -O3 -ffast-math flags, -march=x86-64-v3)",
                   "timing": "host wall clock per step from the request to the last process's answer; grid "
                             f"set-up outside (slowest {r['build_s']:.1f} s)",
                   "same_scheme_engine_rate": "the engine line's same_scheme_as_reference_arm"},
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"each step: {cores} concurrent single-rank processes of the reference's classes, "
                                   f"one RK step (3 solver iterations) each on its own {n}x{n} tile"},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------ modes arm
MODES = {  # name: (side kind, positivity, cylinder, Navier-Stokes shear layer instead of quadrants)
    "periodic": ("BC_PERIODIC", "POSITIVITY_OFF", False, False),
    "transmissive": ("BC_NEUMANN", "POSITIVITY_OFF", False, False),
    "periodic_floors": ("BC_PERIODIC", "POSITIVITY_FLOOR", False, False),
    "transmissive_floors_cylinder": ("BC_NEUMANN", "POSITIVITY_FLOOR", True, False),
    "periodic_navier_stokes": ("BC_PERIODIC", "POSITIVITY_OFF", False, True),
}


def modes_arm(args):
    """Throughput of the row march's feature sets on one grid: a seeded
    four-quadrant state on n^2 cells (default 2048^2), SSP-RK3, Davis HLL, CFL
    0.5, with periodic or transmissive sides, without or with the positivity
    fallbacks and floors, and with a slip-wall cylinder (r = 0.1 at the centre)
    in one mode; the last mode is the periodic Navier-Stokes shear layer (mu =
    1/2000, Pr 0.72) on the same grid.  Each form, each mode: W warm-up steps, K
    timed steps with CUDA events on the engine's stream.  `--mode` runs one mode
    in one form (`--form`, FP32 by default), for a profiler.  One JSON line."""
    import torch

    cfsb = importlib.import_module(PKG)
    wl = importlib.import_module(f"{PKG}.workloads")
    n = args.modes_n
    quads = wl.riemann_quadrants(n, n, seed=3)

    def rate(prec, mode):
        side, pos, cyl, ns = MODES[mode]
        w = wl.shear_layer(n) if ns else quads
        extra = dict(viscous=cfsb.VISCOUS_NS, mu=w.meta["mu"], prandtl=0.72, mach=1.0) if ns else {}
        with cfsb.Solver(n, n, 1.0, 1.0, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                         bc=(getattr(cfsb, side),) * 4, positivity=getattr(cfsb, pos), variant=args.variant,
                         march_rows=args.march_rows, **extra) as s:
            if cyl:
                s.build_circle(0.1, 0.5, 0.5, 400, cfsb.IB_BILINEAR_SLIP)
            s.set_state(w.U0)
            s.advance(args.warmup, cfl=0.5)
            stream = torch.cuda.ExternalStream(s.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            s.advance(args.steps, cfl=0.5)
            e1.record(stream)
            torch.cuda.synchronize()
            return round(n * n * args.steps / (e0.elapsed_time(e1) / 1e3) / 1e6, 1)

    out = {"workload": f"row-march feature sets, four-quadrant state {n}^2, SSP-RK3, Davis HLL, CFL 0.5",
           "steps": args.steps, "warmup": args.warmup, "unit": UNIT}
    if args.mode:
        form = cfsb.FP64 if args.form == "f64" else cfsb.FP32_MIXED
        out[args.mode] = {args.form: rate(form, args.mode)}
    else:
        for mode in MODES:
            out[mode] = {"fp32": rate(cfsb.FP32_MIXED, mode), "fp64": rate(cfsb.FP64, mode)}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--n", type=int, default=4096, help="grid edge (cells) per GPU")
    ap.add_argument("--accuracy-n", type=int, default=1024, help="grid of the FP32-vs-FP64 check (0 = skip)")
    ap.add_argument("--cpu-sample", type=int, default=384, help="grid edge of one CPU-baseline sample")
    ap.add_argument("--workload", choices=["smooth", "batch", "report", "modes"], default="smooth",
                    help="smooth: the headline 4096^2 line; batch: the uneven-batch comparison; report: "
                         "FP32-vs-FP64 accuracy and drift on the other configurations; modes: the row march's "
                         "feature sets on one grid (one JSON line each)")
    ap.add_argument("--cases", type=int, default=512, help="cases of the batch workload")
    ap.add_argument("--batch-cases", type=int, default=512,
                    help="cases of the batch sub-result in the default line (0 = skip)")
    ap.add_argument("--ref-tile", type=int, default=0,
                    help="reference arm: tile edge per host core (0 = tiles summing to n^2 cells)")
    ap.add_argument("--modes-n", type=int, default=2048, help="grid edge of the modes workload")
    ap.add_argument("--mode", choices=list(MODES), default=None, help="modes workload: run this mode only (FP32)")
    ap.add_argument("--variant", type=int, default=0, help="modes workload: stage-kernel variant (0 = default)")
    ap.add_argument("--form", choices=["f32", "f64"], default="f32", help="modes workload with --mode: the form to run")
    ap.add_argument("--march-rows", type=int, default=0,
                    help="modes workload: rows of a row-march work item (0 = chosen per launch)")
    ap.add_argument("--report-parts", default="quadrants,cylinder,shear,batch,convergence",
                    help="report workload: comma-separated parts to run")
    ap.add_argument("--batch-steps", type=int, default=500, help="report workload: steps of the batch comparison")
    ap.add_argument("--conv-max", type=int, default=4096, help="report workload: largest N of the convergence table")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "batch":
        batch_arm(args)
    elif args.workload == "report":
        report_arm(args)
    elif args.workload == "modes":
        modes_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
