"""Supernode-update microbenchmark: batches of dense complex-symmetric fronts.

    python -m aphi_b200.fronts_bench --count 512 --seed 0

Front sizes s are drawn log-uniform in [32, 2048] (seeded), the pivot panel
width is s / 4, entries have real and imaginary parts ~N(0, 1) (symmetric),
and the diagonal is shifted by 2 s. Each front's panel (its first s / 4
columns, all rows) is factorized on the device -- diagonal blocks, panel
rows and the Schur update of the trailing (3 s / 4)^2 block, with the same
plans and kernels as a sparse factorization -- once as complex64 on the
tensor cores (FP32 accumulate) and once as complex128 on the FP64 tensor
path. The trailing block starts at zero, as in the multifrontal method, so
it ends as -L21 D L21^T.

Reported per precision: time for the whole batch, algorithmic TFLOP/s (8 real
flop per complex multiply-add of the pivot steps, sum over fronts of
8 * sum_{j < k} (s - j - 1)(s - j) / 2), the trailing-update kernel's own
throughput and its fraction of the measured peak of the unit it runs on, and
the error of L, D and the Schur update against an FP64 host LDL^T of the
same blocks (on a sample of the fronts: every `--check-every`-th and the
largest).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import aphi_b200 as ab


def front_sizes(count: int, seed: int, lo: int = 32, hi: int = 2048):
    rng = np.random.default_rng(seed)
    s = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int32)
    return s, np.maximum(s // 4, 1).astype(np.int32), rng


def make_panels(rows, widths, rng):
    """Per front the first w columns of a complex-symmetric matrix with
    N(0,1) parts and 2 s added to the diagonal (the block above row w mirrored)."""
    out = []
    for m, w in zip(rows, widths):
        p = rng.standard_normal((m, w)) + 1j * rng.standard_normal((m, w))
        top = np.tril(p[:w])
        p[:w] = top + np.tril(top, -1).T
        p[np.arange(w), np.arange(w)] += 2.0 * m
        out.append(p)
    return out


def pack(fr: ab.Fronts, panels) -> np.ndarray:
    flat = np.zeros(fr.stored, np.complex128)
    for s, p in enumerate(panels):
        o = int(fr.panel_offset[s])
        flat[o:o + p.size] = p.reshape(-1, order="F")
    return flat


def host_ldlt(p: np.ndarray, block: int = 64):
    """Unpivoted complex-symmetric LDL^T of the panel's w columns (blocked,
    right-looking, FP64): returns L (m x w, unit diagonal implied), d, and
    the Schur update L21 D L21^T of the trailing block."""
    m, w = p.shape
    F = p.astype(np.complex128).copy()
    d = np.zeros(w, np.complex128)
    for k0 in range(0, w, block):
        k1 = min(w, k0 + block)
        for k in range(k0, k1):
            d[k] = F[k, k]
            col = F[k + 1:, k] / d[k]
            if k + 1 < k1:
                F[k + 1:, k + 1:k1] -= np.outer(col * d[k], col[:k1 - k - 1])
            F[k + 1:, k] = col
        if k1 < w:
            Lb = F[k1:, k0:k1]
            F[k1:, k1:w] -= (Lb * d[k0:k1]) @ F[k1:w, k0:k1].T
    L21 = F[w:, :]
    return F, d, (L21 * d) @ L21.T


def errors(fr: ab.Fronts, panels, dev_panels: np.ndarray, dev_cb: np.ndarray, sample) -> dict:
    eL, eD, eU = [], [], []
    for s in sample:
        m, w = int(fr.rows[s]), int(fr.widths[s])
        F, d, U = host_ldlt(panels[s])
        o = int(fr.panel_offset[s])
        G = dev_panels[o:o + m * w].reshape(m, w, order="F")
        dd = np.diag(G[:w, :w]).copy()
        low = np.tril(np.ones((m, w), bool), -1)
        eL.append(np.linalg.norm((G - F)[low]) / max(np.linalg.norm(F[low]), 1e-300))
        eD.append(np.linalg.norm(dd - d) / np.linalg.norm(d))
        c = m - w
        if c > 0:
            q = int(fr.cb_offset[s])
            C = dev_cb[q:q + c * c].reshape(c, c, order="F")
            lowc = np.tril(np.ones((c, c), bool))
            eU.append(np.linalg.norm((-C - U)[lowc]) / np.linalg.norm(U[lowc]))
    return {"max_rel_err_L": float(max(eL)), "max_rel_err_D": float(max(eD)),
            "max_rel_err_schur": float(max(eU)) if eU else 0.0, "fronts_checked": len(sample)}


def run(count=512, seed=0, reps=3, check_every=16, lo=32, hi=2048, precisions=("fp32", "fp64")):
    import torch
    rows, widths, rng = front_sizes(count, seed, lo, hi)
    fr = ab.Fronts(rows, widths)
    panels = make_panels(rows, widths, rng)
    flat = torch.from_numpy(pack(fr, panels)).cuda().unsqueeze(0)
    sample = sorted(set(range(0, count, check_every)) | {int(np.argmax(rows))})
    peaks = ab.measure_peaks()
    out = {"config": f"{count} dense complex-symmetric fronts, sizes log-uniform in [{lo}, {hi}] "
                     f"(seed {seed}), panel width size/4, N(0,1) entries + 2*size on the diagonal",
           "count": count, "seed": seed,
           "sizes": {"min": int(rows.min()), "median": int(np.median(rows)), "max": int(rows.max()),
                     "sum_panel_entries": int((rows * widths).sum())},
           "flops_per_batch": fr.info["flops"], "peaks_tflops": peaks}
    for name in precisions:
        prec = ab.PREC_FP32 if name == "fp32" else ab.PREC_FP64
        f = ab.Factor(fr, prec, 1)
        assert f.factorize_fronts(flat)   # warm-up (and workspace)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ms = []
        for _ in range(reps):
            torch.cuda.synchronize()
            ev[0].record()
            f.factorize_fronts(flat)
            ev[1].record()
            torch.cuda.synchronize()
            ms.append(ev[0].elapsed_time(ev[1]))
        f.profile(True)
        f.factorize_fronts(flat)
        kinds = f.profile_read()
        f.profile(False)
        kind = "update_tc" if prec == ab.PREC_FP32 else "update_wide"
        st = fr.plan_stats(1 if prec == ab.PREC_FP32 else 0, flops=True)
        upd_ms = kinds[kind][1]
        upd_tf = st[kind][2] / (upd_ms / 1e3) / 1e12
        if prec == ab.PREC_FP32:
            unit, raw = "tf32_tc_n64", upd_tf * 6        # 24 TF32 MMAs per complex multiply-add of 4
        else:
            unit, raw = "fp64_dmma", upd_tf
        p, c = f.read_fronts(0)
        err = errors(fr, panels, p.cpu().numpy(), c.cpu().numpy(), sample)
        best = min(ms)
        out[name] = {"ms": best, "tflops": fr.info["flops"] / (best / 1e3) / 1e12,
                     "update_kernel": {"kind": kind, "ms": upd_ms, "useful_tflops": upd_tf,
                                       "unit_tflops": raw, "unit": unit, "frac_of_unit_peak": raw / peaks[unit],
                                       "share_of_factorization": upd_ms / sum(v[1] for v in kinds.values())},
                     **err}
        f.close()
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--check-every", type=int, default=16)
    a = ap.parse_args()
    print(json.dumps(run(a.count, a.seed, a.reps, a.check_every)))


if __name__ == "__main__":
    main()
