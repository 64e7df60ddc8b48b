"""Autotuner of the stage-kernel variants (rows marched per warp x warps per
block x occupancy target) of the throughput forms.

For every precision and grid size it times each variant on the smooth periodic
advection workload (SSP-RK3, Davis HLL, on-device CFL dt) with CUDA events on
the engine's stream, and writes the table to ``tuning.json`` next to this file:
``table[precision][size] = {"best": v, "mcell_steps_per_s": {v: rate}}``.
``best_variant(precision, cells)`` reads it back for callers that create
solvers (the benchmark, the batched runner).

Usage (on a GPU): ``python -m 2d_compressible_flow_solver_b200.autotune`` is not
importable by name, so run ``python 2d_compressible_flow_solver_b200/autotune.py
[--sizes 256,1024,4096] [--out path]``.
"""
from __future__ import annotations

import argparse
import importlib
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
TABLE = HERE / "tuning.json"
PRECISIONS = {"f32": 1, "f64": 0}


def _pkg():
    sys.path.insert(0, str(HERE.parent))
    return importlib.import_module(HERE.name), importlib.import_module(f"{HERE.name}.workloads")


def time_variant(cfsb, wl, n: int, prec: int, variant: int, target_ms: float = 60.0):
    import torch

    w = wl.smooth_advection(n)
    with cfsb.Solver(n, n, precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS, bc=(cfsb.BC_PERIODIC,) * 4,
                     variant=variant) as s:
        s.set_state(w.U0)
        s.advance(4, cfl=w.cfl)
        stream = torch.cuda.ExternalStream(s.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # size the timed run to about target_ms
        t0 = time.perf_counter()
        s.advance(2, cfl=w.cfl)
        probe_ms = (time.perf_counter() - t0) * 1e3 / 2
        steps = max(4, min(400, int(target_ms / max(probe_ms, 1e-3))))
        steps += steps % 2
        e0.record(stream)
        s.advance(steps, cfl=w.cfl)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    return n * n * steps / (ms / 1e3) / 1e6


def tune(sizes, precisions, out: Path):
    import torch

    cfsb, wl = _pkg()
    nvar = len(cfsb.variants())
    table = {}
    for pname in precisions:
        prec = PRECISIONS[pname]
        table[pname] = {}
        for n in sizes:
            rates = {}
            for v in range(1, nvar + 1):
                rates[str(v)] = round(time_variant(cfsb, wl, n, prec, v), 1)
            best = max(rates, key=lambda k: rates[k])
            table[pname][str(n)] = {"best": int(best), "mcell_steps_per_s": rates}
            print(pname, n, "best variant", best, rates, flush=True)
    doc = {"device": torch.cuda.get_device_name(0),
           "variants": {str(i + 1): list(v) for i, v in enumerate(cfsb.variants())},
           "workload": "smooth periodic advection n x n, SSP-RK3, Davis HLL, CFL 0.4",
           "table": table}
    out.write_text(json.dumps(doc, indent=1) + "\n")
    return doc


def best_variant(precision: str, cells: int, table_path: Path = TABLE) -> int:
    """Best measured variant for a grid of about `cells` cells (nearest tuned
    size by cell count), as an index of the library's current variant table
    (the table records each variant's shape, so a table tuned against another
    build still maps); 0 (the library default) when no table exists or its best
    shape is not in the library."""
    try:
        doc = json.loads(table_path.read_text())
        rows = doc["table"][precision]
        shapes = doc["variants"]
    except (OSError, KeyError, ValueError):
        return 0
    sizes = sorted(int(k) for k in rows)
    if not sizes:
        return 0
    near = min(sizes, key=lambda n: abs(n * n - cells))
    shape = tuple(shapes.get(str(rows[str(near)]["best"]), ()))
    cfsb, _ = _pkg()
    current = [tuple(v) for v in cfsb.variants()]
    return current.index(shape) + 1 if shape in current else 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="128,256,512,1024,2048,4096")
    ap.add_argument("--precisions", default="f32,f64")
    ap.add_argument("--out", default=str(TABLE))
    a = ap.parse_args()
    tune([int(x) for x in a.sizes.split(",")], a.precisions.split(","), Path(a.out))


if __name__ == "__main__":
    main()
