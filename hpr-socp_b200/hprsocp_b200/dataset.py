"""Dataset runner: solve every CBF file of a folder and write the result
table (run_dataset, src/utils/dataset.jl:4-122).

The table has the reference's columns (name, iter, alg_time, res,
primal_obj, status, iter_4, time_4, iter_6, time_6, power_time) and its two
summary rows: ``SGM10``, the shifted geometric mean exp(mean(log(v + 10)))
- 10 of the iteration counts and times, and ``solved``, the number of runs
whose time stayed under the time limit.  Files already in an existing table
are skipped, so an interrupted run resumes.  The log of every solve is
appended to HPRSOCP_log.txt.

``slots > 0`` solves the files concurrently on one device through the
continuous-batching server instead of one after another; the table is the
same either way (each solve is bit-identical alone and in the mix).
"""
from __future__ import annotations

import csv
import dataclasses
import math
import os
import time
from typing import Callable, Optional

from .cbf import read_cbf_model
from .solver import HPRSOCP_parameters, HPRSOCP_results

COLUMNS = ["name", "iter", "alg_time", "res", "primal_obj", "status", "iter_4", "time_4", "iter_6", "time_6",
           "power_time"]


def sgm10(values) -> float:
    """Shifted geometric mean with shift 10."""
    vals = [float(v) for v in values]
    if not vals:
        return float("nan")
    return math.exp(sum(math.log(v + 10.0) for v in vals) / len(vals)) - 10.0


def _read_table(path: str):
    rows = []
    if os.path.isfile(path):
        with open(path, newline="") as f:
            for r in csv.DictReader(f):
                if r["name"] in ("SGM10", "solved"):
                    continue
                rows.append(r)
    return rows


def _write_table(path: str, rows, time_limit: float):
    iters = [float(r["iter"]) for r in rows]
    times = [float(r["alg_time"]) for r in rows]
    it4 = [float(r["iter_4"]) for r in rows]
    t4 = [float(r["time_4"]) for r in rows]
    it6 = [float(r["iter_6"]) for r in rows]
    t6 = [float(r["time_6"]) for r in rows]
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(COLUMNS)
        for r in rows:
            w.writerow([r[c] for c in COLUMNS])
        w.writerow(["SGM10", sgm10(iters), sgm10(times), "", "", "", sgm10(it4), sgm10(t4), sgm10(it6), sgm10(t6), ""])
        w.writerow(["solved", "", sum(t < time_limit for t in times), "", "", "", "",
                    sum(t < time_limit for t in t4), "", sum(t < time_limit for t in t6), ""])


def _row(name: str, r: HPRSOCP_results, time_limit: float) -> dict:
    return {"name": name, "iter": r.iter, "alg_time": min(r.time, time_limit), "res": r.residuals,
            "primal_obj": r.primal_obj, "status": r.status, "iter_4": r.iter_4,
            "time_4": min(r.time_4, time_limit), "iter_6": r.iter_6, "time_6": min(r.time_6, time_limit),
            "power_time": r.power_time}


def run_dataset(data_path: str, result_path: str, params: Optional[HPRSOCP_parameters] = None, slots: int = 0,
                solve: Optional[Callable] = None):
    """Solve the CBF files of `data_path`; write HPRSOCP_result.csv and
    HPRSOCP_log.txt into `result_path`.  `solve(model, params)` defaults to
    ``optimize``; returns the table rows (without the summary rows)."""
    params = params or HPRSOCP_parameters()
    os.makedirs(result_path, exist_ok=True)
    csv_file = os.path.join(result_path, "HPRSOCP_result.csv")
    log_file = os.path.join(result_path, "HPRSOCP_log.txt")
    rows = _read_table(csv_file)
    done = {r["name"] for r in rows}
    files = [f for f in sorted(os.listdir(data_path)) if f.lower().endswith(".cbf") and f not in done]
    with open(log_file, "a") as log:
        if slots > 0 and solve is None:
            from .serving import Server
            quiet = dataclasses.replace(params, verbose=False)
            with Server(slots=slots, device=params.device_number) as srv:
                tickets = []
                for f in files:
                    tickets.append((f, srv.submit(read_cbf_model(os.path.join(data_path, f)), quiet)))
                for f, t in tickets:
                    r, lat = srv.poll(t)
                    log.write(f"{f}: iter = {r.iter}  time = {r.time:.2e}  residual = {r.residuals:.2e}  "
                              f"primal_obj = {r.primal_obj:.15e}  latency = {lat:.2e}\n")
                    rows.append(_row(f, r, params.time_limit))
            _write_table(csv_file, rows, params.time_limit)
            return rows
        if solve is None:
            from .solver import optimize as solve
        for i, f in enumerate(files, 1):
            print(f"solving the problem {i}: {f}")
            log.write(f"solving the problem {i}: {f}\n")
            t0 = time.perf_counter()
            r = solve(read_cbf_model(os.path.join(data_path, f)), params)
            log.write(f"iter = {r.iter}  time = {r.time:.2e}  residual = {r.residuals:.2e}  "
                      f"primal_obj = {r.primal_obj:.15e}  total = {time.perf_counter() - t0:.2e}\n")
            rows.append(_row(f, r, params.time_limit))
            _write_table(csv_file, rows, params.time_limit)
    return rows
