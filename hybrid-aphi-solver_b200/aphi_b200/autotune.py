"""Per-mesh autotuner for the factorization's schedule.

The supernodal schedule has knobs whose best values depend on the mesh's
front sizes and on the device: how many panels a front's trailing update
applies at once (4-panel groups from `group4_rows` rows up, 2-panel groups
from `group2_rows`, single panels below), which fronts are factored whole in
one CTA (`small_front` rows and fewer), and how far supernodes are relaxed
(`relax_fill`, `relax_max_width`: fewer, wider supernodes at the price of
padded zeros). The permutation is never touched: it is the caller's (the
reference's AMD), and every candidate factors the same matrices to the same
result up to rounding. The panel-group thresholds tuned here are the FP64
plan's; the tensor-core (FP32) plan keeps its own (`tc_group4_rows`,
`tc_group2_rows`), because its grouping sets the FP32 factor's rounding and
so how many refinement steps the stiffer frequencies of a sweep need: a
grouping a few per cent faster to factor cost a whole frequency's FP64
refactorization on the 32^3 sweep.

`tune` builds the analysis for each candidate, times whole factorizations of
the caller's frequencies on the device (CUDA events on the stream the
kernels run on, after one untimed factorization) in FP64 and, when asked,
FP32, and keeps the fastest. It returns the winning analysis (ready to use)
and the table of every trial, which the caller records.
"""
from __future__ import annotations

import itertools
import time

import numpy as np

from . import PREC_FP32, PREC_FP64, Analysis, Factor, default_analysis_options

# The default search: panel-group thresholds and the one-CTA front size.
GRID = {
    "group4_rows": [4096, 8192, 1 << 30],
    "group2_rows": [0, 1024],
    "small_front": [64, 96],
}


def _options(**kw):
    o = default_analysis_options()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _time_factorizations(an, values, precision, reps, stream):
    import torch
    f = Factor(an, precision, values.shape[0])
    try:
        f.factorize(values, stream=stream)   # untimed: allocations, first touches
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            f.factorize(values, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps
    finally:
        f.close()


def tune(row_ptr, col_idx, perm, values, precisions=(PREC_FP64,), grid=None, reps=1, stream=None,
         weights=None):
    """values: complex128 device tensor [batch, nnz] of assembled systems on
    this pattern. Returns (best Analysis, record dict). weights: per-precision
    factors of the score (default 1 each), e.g. the expected number of
    entries each precision will factorize."""
    import torch
    grid = grid or GRID
    keys = list(grid)
    weights = weights or {p: 1.0 for p in precisions}
    trials = []
    best = None
    for combo in itertools.product(*(grid[k] for k in keys)):
        params = dict(zip(keys, combo))
        t0 = time.perf_counter()
        an = Analysis(row_ptr, col_idx, perm, options=_options(**params))
        setup_s = time.perf_counter() - t0
        ms = {}
        for p in precisions:
            ms["fp64" if p == PREC_FP64 else "fp32"] = _time_factorizations(an, values, p, reps, stream)
        score = sum(weights[p] * ms["fp64" if p == PREC_FP64 else "fp32"] for p in precisions)
        trials.append({"params": params, "ms": ms, "score": score, "analysis_s": setup_s,
                       "supernodes": int(an.info["supernodes"]), "stored": int(an.info["stored"])})
        if best is None or score < best[0]:
            if best is not None:
                best[1].close()
            best = (score, an, params)
        else:
            an.close()
        torch.cuda.empty_cache()
    default = next((t for t in trials if all(t["params"][k] == v for k, v in
                                             (("group4_rows", 8192), ("group2_rows", 0), ("small_front", 96))
                                             if k in t["params"])), None)
    record = {"chosen": best[2], "score_ms": best[0], "trials": trials,
              "default_score_ms": default["score"] if default else None,
              "what": "whole factorizations of the given batch, CUDA events, after one untimed run"}
    return best[1], record
