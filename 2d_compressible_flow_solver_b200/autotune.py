"""Autotuner of the stage-kernel variants (rows marched per warp x warps per
block x occupancy target) of the throughput forms.

For every precision and grid size it times each variant on the smooth periodic
advection workload (SSP-RK3, Davis HLL, on-device CFL dt) with CUDA events on
the engine's stream, and writes the table to ``tuning.json`` next to this file:
``table[precision][size] = {"best": v, "mcell_steps_per_s": {v: rate}}``.
``best_variant(precision, cells)`` reads it back for callers that create
solvers (the benchmark, the batched runner).

For the batched engine it also tunes the rows of a work unit (one warp's
segment of a case, marched over that many rows) per case-size bucket, on the
uneven batch itself: a pass of coordinate descent over the buckets, each
trying the candidate rows with the others fixed, writing
``batch_rows[precision] = {"rows": {bucket: rows}, ...}`` beside the variant
table.  (Uniform batches of one size prefer shorter units than the same sizes
among larger cases do, so the sweep runs on the mixed workload.)
``batch_rows_for(precision, nx, ny)`` reads it back: the Batch wrapper gives
every case whose rows are not set the rows of its bucket.

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


# case-size buckets of the batch sweep: upper edges (cells sqrt) of each bucket
BATCH_BUCKETS = (96, 192, 384, 576, 768)


def _bucket(nx: int, ny: int) -> int:
    e = (nx * ny) ** 0.5
    return next((b for b in BATCH_BUCKETS if e <= b), BATCH_BUCKETS[-1])


def time_batch(cfsb, wl, prec: int, rows_of: dict, ncases: int = 512, steps: int = 12) -> float:
    """Mcell-steps/s of the uneven batch (`ncases` cases, nx, ny in 64..768,
    half four-quadrant, half Mach 2-3 cylinder) whose cases of each size
    bucket march work units of rows_of[bucket] rows, timed with CUDA events on
    the batch's stream."""
    import torch

    cases, states = wl.batch_cases(ncases, seed=1)
    cases = [dict(c, rows=rows_of[_bucket(c["nx"], c["ny"])]) for c in cases]
    with cfsb.Batch(cases, precision=prec, positivity=cfsb.POSITIVITY_FLOOR, tuned_rows=False) as b:
        cells, _ = b.info()
        for k, U in enumerate(states):
            b.set_state(k, U)
        b.advance(3, cfl=0.5)
        stream = torch.cuda.ExternalStream(b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.advance(steps, cfl=0.5)
        e1.record(stream)
        torch.cuda.synchronize()
        return cells * steps / (e0.elapsed_time(e1) / 1e3) / 1e6


def tune_batch(precisions, doc: dict, candidates=(16, 32, 64, 96), start: int = 64) -> dict:
    """Adds doc["batch_rows"]: work-unit rows per precision and case-size
    bucket, by one pass of coordinate descent on the uneven batch itself (the
    rows that suit a bucket depend on the cases beside it: units run largest
    case first, so the small cases fill the launch's tail)."""
    cfsb, wl = _pkg()
    out = {}
    for pname in precisions:
        prec = PRECISIONS[pname]
        rows_of = {b: start for b in BATCH_BUCKETS}
        base = time_batch(cfsb, wl, prec, rows_of)
        trials = {}
        for b in BATCH_BUCKETS:
            best_r, best_v = rows_of[b], base
            for r in candidates:
                if r == rows_of[b]:
                    continue
                v = time_batch(cfsb, wl, prec, {**rows_of, b: r})
                trials[f"{b}:{r}"] = round(v, 1)
                if v > best_v * 1.005:  # keep a change only past the run-to-run noise
                    best_r, best_v = r, v
            rows_of[b], base = best_r, best_v
            print(pname, "bucket", b, "rows", best_r, round(best_v, 1), flush=True)
        out[pname] = {"rows": {str(b): rows_of[b] for b in BATCH_BUCKETS}, "mcell_steps_per_s": round(base, 1),
                      "trials": trials}
    doc["batch_rows"] = out
    doc["batch_workload"] = ("the uneven batch: 512 cases, nx, ny in 64..768 step 16, half four-quadrant, half Mach "
                             "2-3 cylinder (slip wall), SSP-RK3, Davis HLL, positivity floors, per-case CFL 0.5; "
                             "buckets by the edge of a square of the case's cells: " + str(BATCH_BUCKETS))
    return doc


def batch_rows_for(precision: str, nx: int, ny: int, table_path: Path = TABLE) -> int:
    """Tuned work-unit rows for a batch case of nx x ny cells (its size
    bucket); 0 (the library default) without a table."""
    try:
        rows = json.loads(table_path.read_text())["batch_rows"][precision]["rows"]
    except (OSError, KeyError, ValueError, TypeError):
        return 0
    return int(rows.get(str(_bucket(nx, ny)), 0))


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
    ap.add_argument("--batch", type=int, default=1, help="1: also tune the batch work-unit rows per case size")
    a = ap.parse_args()
    out = Path(a.out)
    doc = tune([int(x) for x in a.sizes.split(",")], a.precisions.split(","), out)
    if a.batch:
        tune_batch(a.precisions.split(","), doc)
        out.write_text(json.dumps(doc, indent=1) + "\n")


if __name__ == "__main__":
    main()
