"""Refinement study: how far up the frequency sweep an FP32 factor still
preconditions the cylinder systems, and at what cost.

    python -m aphi_b200.refine_study --cells 32 --restart 40 --max-iters 200

For each frequency of the 16-point sweep (50 Hz .. 1 MHz) it factors the
system once in FP64 and once in FP32 (tensor cores, two-piece split) and
reports, as one JSON line per frequency:
  * rho: an estimate of the spectral radius of I - M^-1 A (12 power
    iterations), M the FP32 factor -- plain refinement converges only when it
    is below 1, and cond(A) * eps(FP32) is its scale;
  * COCG (the library's refinement, aphi_solve_refined): iterations, final
    relative residual, forward error against the FP64 solution;
  * right-preconditioned flexible GMRES(restart) in FP64 with classical
    Gram-Schmidt twice, the FP32 factor as preconditioner: iterations to
    relative residual 1e-14, backward error, forward error, device time.
Every matrix-vector product is the library's SpMV (aphi_spmv), every
preconditioner application the library's FP32 solve; only the Krylov basis
arithmetic (inner products, updates) is plain tensor algebra here.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import aphi_b200 as ab


def fgmres(A, M, b, x0, restart, max_iters, tol):
    """Right-preconditioned flexible GMRES with CGS2; returns x, iterations,
    the relative residual after each restart."""
    import torch
    bn = torch.linalg.vector_norm(b).item()
    x = x0
    its = 0
    hist = []
    while True:
        r = b - A(x)
        beta = torch.linalg.vector_norm(r).item()
        hist.append(beta / bn)
        if beta / bn <= tol or its >= max_iters:
            return x, its, hist
        V = [r / beta]
        Z = []
        H = np.zeros((restart + 1, restart), np.complex128)
        g = np.zeros(restart + 1, np.complex128)
        g[0] = beta
        cs = np.zeros(restart, np.complex128)
        sn = np.zeros(restart, np.complex128)
        jd = 0
        for j in range(restart):
            z = M(V[j])
            Z.append(z)
            w = A(z)
            Vm = torch.stack(V)
            h = torch.conj(Vm) @ w
            w = w - Vm.T @ h
            h2 = torch.conj(Vm) @ w
            w = w - Vm.T @ h2
            hj = (h + h2).cpu().numpy()
            hn = torch.linalg.vector_norm(w).item()
            H[:j + 1, j] = hj
            H[j + 1, j] = hn
            for i in range(j):
                t = np.conj(cs[i]) * H[i, j] + np.conj(sn[i]) * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = np.hypot(abs(H[j, j]), abs(H[j + 1, j]))
            cs[j], sn[j] = H[j, j] / den, H[j + 1, j] / den
            H[j, j], H[j + 1, j] = den, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = np.conj(cs[j]) * g[j]
            its += 1
            jd = j + 1
            if hn > 0:
                V.append(w / hn)
            if abs(g[j + 1]) / bn <= 0.3 * tol or its >= max_iters or hn == 0:
                break
        y = np.linalg.solve(np.triu(H[:jd, :jd]), g[:jd])
        x = x + torch.stack(Z).T @ torch.from_numpy(y).to(x.device)


def main() -> None:
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=32)
    ap.add_argument("--restart", type=int, default=40)
    ap.add_argument("--max-iters", type=int, default=200)
    ap.add_argument("--index", default="", help="comma list of sweep indices (default: all 16)")
    a = ap.parse_args()
    w = ab.Workload.cylinder(a.cells)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    omegas = 2 * np.pi * np.geomspace(50.0, 1.0e6, 16)
    idx = [int(v) for v in a.index.split(",")] if a.index else list(range(16))
    f64 = ab.Factor(an)
    f32 = ab.Factor(an, precision=ab.PREC_FP32)
    f32.set_tc_split(2)
    for k in idx:
        vals, rhs = asm.refill(omegas[k])
        b = rhs[0].clone()
        bn = torch.linalg.vector_norm(b).item()
        amax = torch.abs(vals).max().item()

        def A(x):
            return ab.spmv(an, vals, x.unsqueeze(0))[0]

        def M(v):
            return f32.solve(v.unsqueeze(0))[0]

        assert f64.factorize(vals)
        x64 = f64.solve(rhs)[0]
        assert f32.factorize(vals)
        xc, itc, _, convc = f32.solve_refined(vals, rhs, tol=1e-16, rtol=1e-14, max_iters=a.max_iters)
        g = torch.Generator(device="cuda").manual_seed(1)
        v = torch.randn(an.n, dtype=torch.complex128, device="cuda", generator=g)
        v /= torch.linalg.vector_norm(v)
        rho = 0.0
        for _ in range(12):
            v2 = v - M(A(v))
            rho = torch.linalg.vector_norm(v2).item()
            v = v2 / max(rho, 1e-300)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x, its, hist = fgmres(A, M, b, M(b), a.restart, a.max_iters, 1e-14)
        torch.cuda.synchronize()
        t_gm = time.perf_counter() - t0
        res = torch.linalg.vector_norm(b - A(x)).item()
        nx64 = torch.linalg.vector_norm(x64).item()
        rec = {"cells": a.cells, "sweep_index": k, "f_hz": omegas[k] / (2 * np.pi), "rho_I_minus_MinvA": rho,
               "cocg": {"iters": int(itc[0, 0]), "converged": bool(convc),
                        "rel_residual": torch.linalg.vector_norm(b - A(xc[0])).item() / bn,
                        "fwd_err_vs_fp64": torch.linalg.vector_norm(xc[0] - x64).item() / nx64},
               "fgmres": {"restart": a.restart, "iters": its, "converged": hist[-1] <= 1e-14,
                          "rel_residual": res / bn,
                          "backward_error": res / (amax * torch.linalg.vector_norm(x).item() + bn),
                          "fwd_err_vs_fp64": torch.linalg.vector_norm(x - x64).item() / nx64, "seconds": t_gm,
                          "restart_history": hist}}
        print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
