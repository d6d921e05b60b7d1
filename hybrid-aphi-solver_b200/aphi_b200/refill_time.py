"""Time the device assembly (element fill + scatter) of a frequency batch --
the command the assembly profiles are taken with.

    python -m aphi_b200.refill_time 32 16

Builds the cylinder-in-box workload and its device assembly, refills the
first `nf` of the sweep's log-spaced frequencies (50 Hz .. 1 MHz) once
untimed, then five times into the same buffers, and prints one JSON line
with the mean device time per refill (CUDA events on the launching stream).
"""
from __future__ import annotations

import json
import sys

import numpy as np

import aphi_b200 as ab


def main() -> None:
    import torch
    cells = int(sys.argv[1]) if len(sys.argv) > 1 else 32
    nf = int(sys.argv[2]) if len(sys.argv) > 2 else 16
    w = ab.Workload.cylinder(cells)
    asm = ab.Assembly(ab.workload_arrays(w))
    om = 2 * np.pi * np.geomspace(50.0, 1.0e6, nf)
    v, r = asm.refill(om)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(5):
        asm.refill(om, values=v, rhs=r)
    b.record()
    torch.cuda.synchronize()
    print(json.dumps({"cells": cells, "frequencies": nf, "ms_per_refill": a.elapsed_time(b) / 5,
                      "num_terms": asm.num_terms, "nnz": asm.nnz}))


if __name__ == "__main__":
    main()
