"""The multiply-connected large case: the copper torus (major radius 0.25,
minor 0.04) in the unit box at n^3 cells x 6 Kuhn tets, one 1 A internal
current port on its cut, and a sweep of log-spaced frequencies 50 Hz - 10 kHz.
The mixed path (FP32 factorization on the tensor cores, FP64 refinement,
automatic FP64 refactorization where the refinement stalls, the refactorized
entries refined too) against the plain FP64 path (the drop-in: factorize and
solve, no refinement), every solve complex128 in and out, factor batches sized to the
device memory.

    python -m aphi_b200.torus_bench [--cells 48] [--nfreq 8] [--steps 1] [--budget-gb 150]

prints one JSON object: the problem's sizes, host setup times, both paths'
solves/s over the timed sweeps (CUDA events on the solving stream), the
precision each frequency ended in, backward errors and relative residuals,
and the port impedance V / I per frequency. The mixed path's acceptance is
the plain FP64 path's backward error (see run()).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

import aphi_b200 as ab


def sweep_timing(solver, omegas, steps, stream):
    solver.solve(omegas, stream=stream)  # warm-up: allocations, and the mixed path learns where FP32 stalls
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        out = solver.solve(omegas, stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, out


def run(cells: int, nfreq: int, steps: int, budget_gb: float, f_lo: float, f_hi: float) -> dict:
    t0 = time.perf_counter()
    w = ab.Workload.torus(cells)
    t1 = time.perf_counter()
    perm = ab.amd_ordering(w.row_ptr, w.col_idx)
    t2 = time.perf_counter()
    an = ab.Analysis(w.row_ptr, w.col_idx, perm)
    t3 = time.perf_counter()
    asm = ab.Assembly(ab.workload_arrays(w))
    info = an.info
    fb = info["factor_bytes_fp64"]
    budget = budget_gb * 1e9
    # Plain FP64: as many entries per factorization as the budget holds. Mixed:
    # the FP32 factor (half the bytes) takes 60 %, the FP64 fallback factor 40 %.
    fp64_batch = int(max(1, min(nfreq, budget // fb)))
    fp32_batch = int(max(1, min(nfreq, (0.6 * budget) // (fb / 2))))
    fallback_batch = int(max(1, min(nfreq, (0.4 * budget) // fb)))
    omegas = 2 * np.pi * np.geomspace(f_lo, f_hi, nfreq)
    stream = torch.cuda.current_stream()
    k = int(w.port_row[0])
    current = complex(w.port_amplitude[0], w.port_amplitude[1])

    # The only source is the port's r * I in one row, so ||b|| is tiny next to
    # ||A|| ||x||: the relative residual of any FP64 solve floors near
    # eps ||A|| ||x|| / ||b|| (1e-5 at 32^3), and the backward error is the
    # yardstick. The plain FP64 path runs first; the mixed path then accepts an
    # FP32 entry whose refined backward error is within 2x of FP64's worst.
    fp64 = ab.SweepSolver(an, asm, nfreq, "fp64", fp64_batch=fp64_batch)
    ms_64, (x64, vals64, rhs64, _) = sweep_timing(fp64, omegas, steps, stream)
    res_64 = ab.residuals(an, vals64, x64, rhs64)
    z_64 = x64[:, k].cpu().numpy() / current
    fp64.close()
    del fp64, x64, vals64, rhs64
    torch.cuda.empty_cache()
    tol = 2.0 * float(res_64[:, 0, 1].max())

    mixed = ab.SweepSolver(an, asm, nfreq, "mixed", fp64_batch=fallback_batch, fp32_batch=fp32_batch,
                           fp64_refine=True, rtol=1.0, tol=tol)
    ms_mixed, (x, vals, rhs, reports) = sweep_timing(mixed, omegas, steps, stream)
    res_mixed = ab.residuals(an, vals, x, rhs)
    z_mixed = x[:, k].cpu().numpy() / current
    precisions = [r["precision"] for r in reports]
    iters = [int(r.get("iterations", 0)) for r in reports]
    mixed.close()
    del mixed, x, vals, rhs
    torch.cuda.empty_cache()

    return {
        "config": {"workload": f"torus {cells}^3 cells, 1 A internal current port", "cells": cells,
                   "tets": w.num_tets, "unknowns": an.n, "nnz_upper": an.nnz, "nnz_L": int(info["nnz_l"]),
                   "stored": int(info["stored"]), "max_front_rows": int(info["max_rows"]),
                   "flops_per_factorization": info["flops"], "factor_bytes_fp64": fb,
                   "frequencies_hz": [float(o / (2 * np.pi)) for o in omegas], "data": "synthetic"},
        "host_setup_s": {"workload": t1 - t0, "amd": t2 - t1, "analysis": t3 - t2},
        "mixed": {"solves_per_s": nfreq / (ms_mixed / 1000.0), "ms_per_sweep": ms_mixed,
                  "fp32_batch": fp32_batch, "fp64_fallback_batch": fallback_batch, "precision": precisions,
                  "refinement_iterations": iters, "backward_error_target": tol,
                  "max_backward_error": float(res_mixed[:, 0, 1].max()),
                  "max_relative_residual": float(res_mixed[:, 0, 0].max())},
        "fp64": {"solves_per_s": nfreq / (ms_64 / 1000.0), "ms_per_sweep": ms_64, "batch": fp64_batch,
                 "max_backward_error": float(res_64[:, 0, 1].max()),
                 "max_relative_residual": float(res_64[:, 0, 0].max())},
        "speedup_mixed_over_fp64": ms_64 / ms_mixed,
        "port_impedance_ohm": [[float(z.real), float(z.imag)] for z in z_64],
        "max_impedance_difference": float(np.max(np.abs(z_mixed - z_64) / np.abs(z_64))),
        "steps": steps,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--cells", type=int, default=48)
    ap.add_argument("--nfreq", type=int, default=8)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--f-lo", type=float, default=50.0)
    ap.add_argument("--f-hi", type=float, default=1e4)
    a = ap.parse_args()
    print(json.dumps(run(a.cells, a.nfreq, a.steps, a.budget_gb, a.f_lo, a.f_hi)))


if __name__ == "__main__":
    main()
