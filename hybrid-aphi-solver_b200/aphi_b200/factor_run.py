"""Factorize one frequency batch of the cylinder-in-box and print the device
time of each kernel kind -- the command the kernel profiles are taken with.

    python -m aphi_b200.factor_run --cells 24 --batch 1 --precision 64

It builds the workload, the reference's AMD ordering and the supernodal
analysis on the host, assembles `batch` log-spaced frequencies on the device,
factorizes them `--reps` times and prints one JSON line: per kind the launches
and milliseconds of the last factorization, the useful Schur-update flops of
the plan, and the whole factorization's time. With `--solves N` it then times
N solves of the batch's right-hand sides (CUDA events, after one untimed
solve), one more with per-kind timing, and the solves' algorithmic factor
traffic (2 nnz(L) values per entry) per millisecond.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

import aphi_b200 as ab


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=24)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--precision", type=int, default=64, choices=[32, 64])
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--f-lo", type=float, default=50.0)
    ap.add_argument("--f-hi", type=float, default=1.0e3)
    ap.add_argument("--simt", action="store_true", help="FP32 on the SIMT kernels instead of tcgen05")
    ap.add_argument("--tc-split", type=int, default=3, choices=[2, 3],
                    help="TF32 pieces per operand in the tensor-core update")
    ap.add_argument("--solves", type=int, default=0, help="also time this many solves of the batch")
    a = ap.parse_args()
    import torch
    if a.simt:
        os.environ["APHI_NO_TC"] = "1"
    w = ab.Workload.cylinder(a.cells)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.geomspace(a.f_lo, a.f_hi, a.batch))
    f = ab.Factor(an, precision=a.precision, batch=a.batch)
    if a.precision == 32:
        f.set_tc_split(a.tc_split)
    ok = True
    ms = 0.0
    kinds = {}
    for r in range(a.reps):
        f.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ok = f.factorize(vals) and ok
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        kinds = f.profile_read()
    plan = an.plan_stats(1 if a.precision == 32 and not a.simt else 0, flops=True)
    out = {"cells": a.cells, "batch": a.batch, "precision": a.precision, "tensor_cores": a.precision == 32 and not a.simt,
           "tc_split": a.tc_split if a.precision == 32 else None,
           "ok": ok, "factorize_ms": ms, "flops_per_factorization": an.info["flops"],
           "kinds": {k: {"launches": n, "ms": t, "useful_flops": plan.get(k, (0, 0, 0.0))[2] * a.batch,
                         "tflops": (plan.get(k, (0, 0, 0.0))[2] * a.batch / (t / 1000.0) / 1e12) if t else None}
                     for k, (n, t) in kinds.items()}}
    if a.solves > 0:
        f.profile(False)
        f.solve(rhs)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.solves):
            f.solve(rhs)
        e1.record()
        torch.cuda.synchronize()
        sms = e0.elapsed_time(e1) / a.solves
        f.profile(True, ["fwd_gather", "fwd_diag", "fwd_update", "bwd_update", "bwd_diag"])
        f.solve(rhs)
        torch.cuda.synchronize()
        value_bytes = 16 if a.precision == 64 else 8
        traffic = 2.0 * an.info["nnz_l"] * value_bytes * a.batch
        out["solve"] = {"ms": sms, "factor_gb_per_s": traffic / sms / 1e6,
                        "kinds": {k: {"launches": n, "ms": t} for k, (n, t) in f.profile_read().items()}}
        f.profile(False)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
