"""Extended-precision checks shared by the solve tests: A x for the
upper-stored matrix in numpy clongdouble, and x*, a solution refined with
extended-precision residuals and corrections from an FP64 factor."""
import numpy as np
import torch


def spmv_extended(rp, ci, v, x):
    """A x for the upper-stored A in extended precision (numpy clongdouble)."""
    n = rp.size - 1
    vl = v.astype(np.clongdouble)
    xl = x.astype(np.clongdouble)
    rows = np.repeat(np.arange(n), np.diff(rp))
    y = np.zeros(n, np.clongdouble)
    np.add.at(y, rows, vl * xl[ci])
    off = ci != rows
    np.add.at(y, ci[off], vl[off] * xl[rows[off]])
    return y


def refined_solution(factor, rp, ci, v, b, x, steps=6):
    """x* : x refined with residuals in extended precision and corrections
    from the FP64 factor -- a reference solution accurate well beyond what a
    plain FP64 solve of an ill-conditioned system gives."""
    for _ in range(steps):
        r = np.array(b.astype(np.clongdouble) - spmv_extended(rp, ci, v, x), np.complex128)
        dx = factor.solve(torch.from_numpy(r).cuda().unsqueeze(0))[0].cpu().numpy()
        x = np.array(x.astype(np.clongdouble) + dx.astype(np.clongdouble), np.complex128)
    return x


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)
