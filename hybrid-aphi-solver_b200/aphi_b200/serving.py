"""Serving loop: (mesh, frequency, port excitations) requests solved as they
arrive, with continuous batching on one GPU.

    python -m aphi_b200.serving --rate 200 --duration 10 --precision mixed

A request names a cylinder-in-box mesh (N cells a side), one frequency and
1-8 voltage excitations of the top port (unit-magnitude phasors); its answer
is the field for every excitation, to relative residual <= 1e-10.

How it runs:
  * Per-mesh state is cached on the device: the workload, the reference's AMD
    ordering, the supernodal analysis and the assembly (slot -> term lists),
    built once per mesh (`MeshCache`).
  * Requests wait in one FIFO queue per mesh. Worker threads, each with its
    own CUDA stream, repeatedly take the mesh whose oldest request has waited
    longest and form a batch from up to `max_batch` of its waiting requests:
    one frequency-batched refill, one batched factorization and one refined
    multi-RHS solve. Requests that arrive while batches run are picked up by
    the next batch of their mesh (continuous batching); batches of different
    meshes run at the same time on different streams and overlap on the
    device. A mesh is handled by one worker at a time, because its analysis
    owns the contribution-block workspace its factorizations use.
  * Admission by HBM footprint: each resident mesh keeps its factors (FP64,
    and FP32 in mixed mode) allocated at a batch capacity chosen so that all
    of them, with their workspaces and solve buffers, fit within
    `hbm_budget`; batches never allocate, so they never stall other streams
    on a device-wide free. A request for a mesh without a resident analysis,
    or with more excitations than the buffers hold, is rejected.
  * Right-hand sides: the right-hand side is linear in the prescribed port
    voltage, so each excitation is V times the 1 V right-hand side of the
    request's frequency.
  * precision="mixed": FP32 factorization plus FP64 preconditioned COCG;
    entries whose refinement stalls are refactorized in FP64, and the mesh
    remembers the lowest frequency at which that happened so that later
    requests at or above it go to FP64 directly. Each mesh is calibrated
    first (`MeshCache.calibrate`): where one FP32-refined request costs more
    than one FP64 request, the mesh's requests all go to FP64, so the mixed
    server is never slower than the plain one. precision="fp64": FP64
    factorization and direct solve (the plain drop-in path).
  * Load shedding (`max_queue`): a request that finds its mesh's queue full
    is rejected at once, so an offered load beyond the device's rate gives a
    bounded queue and honest latencies for the requests served.

Each request's result depends only on its own system: batches never mix the
arithmetic of different entries, so a request gives the same answer alone and
in a mix (the tests check this).
"""
from __future__ import annotations

import argparse
import collections
import json
import threading
import time
from dataclasses import dataclass, field

import numpy as np

import aphi_b200 as ab


@dataclass
class Request:
    rid: int
    cells: int
    omega: float
    voltages: np.ndarray          # complex, one per right-hand side
    arrival: float = 0.0          # seconds since the trace started
    # filled in by the server
    x: np.ndarray | None = None   # [nrhs, n] complex128 on the host
    admitted: float = 0.0
    done: float = 0.0
    precision: str = ""
    residual: float = float("nan")
    backward_error: float = float("nan")
    batch_size: int = 0
    error: str = ""

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class MeshCache:
    """Device-resident per-mesh state: analysis, assembly and the frequency
    above which FP32 refinement is known to stall on this mesh."""

    def __init__(self, cells: int):
        self.cells = cells
        w = ab.Workload.cylinder(cells)
        self.analysis = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
        self.assembly = ab.Assembly(ab.workload_arrays(w))
        self.n = self.analysis.n
        self.nnz = self.analysis.nnz
        info = self.analysis.info
        self.stored, self.cb_pool = int(info["stored"]), int(info["cb_pool"])
        self.stall_omega = None
        self.lock = threading.Lock()
        # the analysis uploads its schedule when its first factor is made
        ab.Factor(self.analysis, ab.PREC_FP64, 1).close()
        self.fp32_pays = True     # set by calibrate()
        self.calibration = None

    def calibrate(self, rtol: float = 1e-12, tol: float = 1e-15, max_iters: int = 40) -> dict:
        """Times one request's worth of work both ways on this mesh, at the
        low end of the band where FP32 refinement converges (50 Hz): FP64
        factorization + direct solve, and FP32 factorization + FP64-refined
        solve. Where the mixed path is not the faster one (small meshes, whose
        factorizations are cheap next to the refinement's solves), mixed
        serving routes this mesh's requests to FP64, so mixed never serves
        slower than plain FP64."""
        import torch
        vals, rhs = self.assembly.refill(2 * np.pi * 50.0)
        ms = {}
        for name, prec in (("fp64", ab.PREC_FP64), ("fp32_ir", ab.PREC_FP32)):
            f = ab.Factor(self.analysis, prec, 1)
            if prec == ab.PREC_FP32:
                f.set_tc_split(2)
            for rep in range(2):      # the first pass is untimed
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                f.factorize(vals)
                if prec == ab.PREC_FP64:
                    f.solve(rhs)
                else:
                    f.solve_refined(vals, rhs, tol=tol, rtol=rtol, max_iters=max_iters)
                e1.record()
                torch.cuda.synchronize()
                ms[name] = e0.elapsed_time(e1)
            f.close()
        self.fp32_pays = ms["fp32_ir"] < ms["fp64"]
        self.calibration = ms
        return ms

    def footprint(self, batch: int, nrhs: int, precision: int) -> int:
        """Device bytes a batch needs: the factor (panels), the contribution
        block workspace, and solve / refinement vectors."""
        elem = 16 if precision == ab.PREC_FP64 else 8
        return int((self.stored + self.cb_pool) * batch * elem + 14 * self.n * nrhs * batch * 16
                   + 3 * self.nnz * batch * 16)


@dataclass
class _Worker:
    index: int
    stream: object


class Server:
    def __init__(self, meshes: dict, precision: str = "mixed", workers: int = 2, max_batch: dict | None = None,
                 hbm_budget: float = 150e9, rtol: float = 1e-12, tol: float = 1e-15, max_iters: int = 40,
                 target_residual: float = 1e-10, max_queue: int | None = None):
        import torch
        if precision not in ("mixed", "fp64"):
            raise ab.InvalidArgument(ab.ERR_BAD_SHAPE, f"Server: precision {precision!r} is not mixed or fp64")
        self.meshes = meshes
        self.precision = precision
        self.rtol, self.tol, self.max_iters = rtol, tol, max_iters
        self.target = target_residual
        self.budget = hbm_budget
        # Load shedding: a request that finds this many requests of its mesh
        # already waiting is rejected at once rather than queued without bound
        # (None: no bound).
        self.max_queue = max_queue
        self.max_batch = dict(max_batch or {c: (4 if c >= 32 else 8 if c >= 24 else 16) for c in meshes})
        # Admission by HBM footprint: every mesh keeps an FP64 factor (and an
        # FP32 one in mixed mode) of its batch capacity resident, allocated
        # here once; capacities are halved, largest mesh first, until all of
        # them fit the budget.
        precs = [ab.PREC_FP64] + ([ab.PREC_FP32] if precision == "mixed" else [])

        def total():
            return sum(m.footprint(self.max_batch[c], 8, p) for c, m in meshes.items() for p in precs)

        for c in sorted(meshes, reverse=True):
            while total() > hbm_budget and self.max_batch[c] > 1:
                self.max_batch[c] //= 2
        self.footprint = total()
        self.factors = {(c, p): ab.Factor(m.analysis, p, self.max_batch[c]) for c, m in meshes.items() for p in precs}
        for (c, p), f in self.factors.items():
            if p == ab.PREC_FP32:
                f.set_tc_split(2)     # hh + hl + lh: the refinement needs no more iterations than with 3
        self.queues = {c: collections.deque() for c in meshes}
        self.busy = set()
        self.cv = threading.Condition()
        self.finished = []
        self.rejected = []
        self.closed = False
        self.t0 = time.perf_counter()
        self.workers = [_Worker(k, torch.cuda.Stream()) for k in range(workers)]
        self.threads = [threading.Thread(target=self._run, args=(wk,), daemon=True) for wk in self.workers]
        self.errors = []
        for t in self.threads:
            t.start()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ------------------------------------------------------------ admission
    def submit(self, req: Request) -> None:
        m = self.meshes.get(req.cells)
        nrhs = len(req.voltages)
        with self.cv:
            if m is None or not 1 <= nrhs <= 8:
                req.error = "rejected: no resident analysis for this mesh, or not 1-8 excitations"
                self.rejected.append(req)
                return
            if self.max_queue is not None and len(self.queues[req.cells]) >= self.max_queue:
                req.error = "shed: the mesh's queue is full"
                self.rejected.append(req)
                return
            self.queues[req.cells].append(req)
            self.cv.notify_all()

    def close(self) -> None:
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        for t in self.threads:
            t.join()
        for f in self.factors.values():
            f.close()
        self.factors = {}
        if self.errors:
            raise self.errors[0]

    def _pick(self):
        """Under the lock: the free mesh whose oldest request has waited
        longest; pops up to its batch capacity of requests."""
        best = None
        for c, q in self.queues.items():
            if q and c not in self.busy and (best is None or q[0].arrival < self.queues[best][0].arrival):
                best = c
        if best is None:
            return None
        q = self.queues[best]
        batch = [q.popleft() for _ in range(min(self.max_batch[best], len(q)))]
        self.busy.add(best)
        return best, batch

    def _run(self, wk: _Worker) -> None:
        import torch
        torch.cuda.set_device(0)
        while True:
            with self.cv:
                got = None
                while got is None:
                    got = self._pick()
                    if got is None:
                        if self.closed and not any(self.queues.values()):
                            return
                        self.cv.wait(timeout=0.05)
            cells, batch = got
            t_admit = self.now()
            try:
                with torch.cuda.stream(wk.stream):
                    self._solve_batch(wk, self.meshes[cells], batch)
            except Exception as e:  # surfaced by close()
                for r in batch:
                    r.error = f"{type(e).__name__}: {e}"
                self.errors.append(e)
            t_done = self.now()
            with self.cv:
                for r in batch:
                    r.admitted, r.done, r.batch_size = t_admit, t_done, len(batch)
                    self.finished.append(r)
                self.busy.discard(cells)
                self.cv.notify_all()

    # ------------------------------------------------------------ the work
    def _solve_batch(self, wk: _Worker, m: MeshCache, batch: list) -> None:
        import torch
        stream = wk.stream
        with m.lock:
            om = np.array([r.omega for r in batch])
            nb = len(batch)
            nrhs = max(len(r.voltages) for r in batch)
            vals, rhs1 = m.assembly.refill(om, stream=stream)
            # excitations: V * (the 1 V right-hand side); short lists repeat their last
            V = np.ones((nb, nrhs), np.complex128)
            for i, r in enumerate(batch):
                V[i, :len(r.voltages)] = r.voltages
                V[i, len(r.voltages):] = r.voltages[-1]
            Vd = torch.from_numpy(V).to(device=vals.device, non_blocking=False)
            b = Vd[:, :, None] * rhs1[:, None, :]
            x = torch.empty_like(b)
            prec_of = ["fp64"] * nb
            todo = list(range(nb))
            if self.precision == "mixed" and m.fp32_pays:
                fp32 = [i for i in range(nb) if m.stall_omega is None or om[i] < m.stall_omega]
                todo = [i for i in range(nb) if i not in fp32]
                if fp32:
                    f = self.factors[(m.cells, ab.PREC_FP32)]
                    sel = torch.tensor(fp32, device=vals.device)
                    v, bb = vals.index_select(0, sel), b.index_select(0, sel).contiguous()
                    f.set_batch(len(fp32))
                    f.factorize(v, 10, 0.0, stream=stream)
                    xs, _, _, _ = f.solve_refined(v, bb, tol=self.tol, rtol=self.rtol, max_iters=self.max_iters,
                                                  stream=stream)
                    res = ab.residuals(m.analysis, v, xs, bb, stream=stream)
                    x.index_copy_(0, sel, xs)
                    for q, i in enumerate(fp32):
                        if (res[q, :, 0] <= self.rtol).all():
                            prec_of[i] = "fp32"
                        else:
                            todo.append(i)
                            with self.cv:
                                if m.stall_omega is None or om[i] < m.stall_omega:
                                    m.stall_omega = float(om[i])
            if todo:
                todo.sort()
                f = self.factors[(m.cells, ab.PREC_FP64)]
                sel = torch.tensor(todo, device=vals.device)
                v, bb = vals.index_select(0, sel), b.index_select(0, sel).contiguous()
                f.set_batch(len(todo))
                f.factorize(v, 10, 0.0, stream=stream)
                xs = f.solve(bb, stream=stream)
                x.index_copy_(0, sel, xs)
            res = ab.residuals(m.analysis, vals, x, b, stream=stream)
            xh = x.cpu().numpy()
        for i, r in enumerate(batch):
            k = len(r.voltages)
            r.x = xh[i, :k].copy()
            r.residual = float(res[i, :k, 0].max())
            r.backward_error = float(res[i, :k, 1].max())
            r.precision = prec_of[i]


def make_trace(rate: float, duration: float, cells=(8, 12, 16, 24, 32), f_lo: float = 50.0, f_hi: float = 1e8,
               max_rhs: int = 8, seed: int = 0) -> list:
    """Poisson arrivals at `rate` per second for `duration` seconds; each
    request a uniform mesh, a log-uniform frequency and 1..max_rhs unit
    phasors at uniform random phase."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        c = int(rng.choice(cells))
        f = float(np.exp(rng.uniform(np.log(f_lo), np.log(f_hi))))
        k = int(rng.integers(1, max_rhs + 1))
        v = np.exp(1j * rng.uniform(0, 2 * np.pi, size=k))
        out.append(Request(len(out), c, 2 * np.pi * f, v, arrival=t))
    return out


def run_trace(server: Server, trace: list) -> dict:
    """Feed the trace in real time (each request submitted at its arrival
    time), wait for every answer, return latency / throughput figures."""
    t0 = server.now()
    for r in trace:
        delay = r.arrival - (server.now() - t0)
        if delay > 0:
            time.sleep(delay)
        r.arrival = server.now()
        server.submit(r)
    with server.cv:
        while len(server.finished) + len(server.rejected) < len(trace) and not server.errors:
            server.cv.wait(timeout=0.1)
    done = [r for r in server.finished if not r.error]
    lat = np.array([r.latency for r in done]) if done else np.zeros(1)
    span = max(r.done for r in done) - min(r.arrival for r in trace) if done else 1.0
    rhs = sum(len(r.voltages) for r in done)
    return {"requests": len(trace), "completed": len(done), "rejected": len(server.rejected),
            "shed": sum(1 for r in server.rejected if r.error.startswith("shed")),
            "failed": sum(1 for r in server.finished if r.error),
            "solves_per_s": len(done) / span, "rhs_per_s": rhs / span, "span_s": span,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "max_residual": float(max((r.residual for r in done), default=0.0)),
            "max_backward_error": float(max((r.backward_error for r in done), default=0.0)),
            "above_target": [[r.cells, r.omega / (2 * np.pi), r.residual, r.backward_error, r.batch_size, r.precision]
                             for r in done if not r.residual <= server.target][:20],
            "fp32_requests": sum(r.precision == "fp32" for r in done),
            "mean_batch": float(np.mean([r.batch_size for r in done])) if done else 0.0,
            "per_mesh": {c: {"completed": sum(1 for r in done if r.cells == c),
                             "p50_ms": float(np.percentile([r.latency for r in done if r.cells == c] or [0], 50) * 1e3),
                             "p99_ms": float(np.percentile([r.latency for r in done if r.cells == c] or [0], 99) * 1e3)}
                         for c in server.meshes}}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--cells", default="8,12,16,24,32")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--f-hi", type=float, default=1e8)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-queue", type=int, default=0, help="per-mesh queue bound (0: unbounded)")
    a = ap.parse_args()
    cells = [int(c) for c in a.cells.split(",")]
    t0 = time.perf_counter()
    meshes = {c: MeshCache(c) for c in cells}
    calib = {}
    if a.precision == "mixed":
        calib = {c: dict(m.calibrate(), fp32_pays=m.fp32_pays) for c, m in meshes.items()}
    setup = time.perf_counter() - t0
    trace = make_trace(a.rate, a.duration, cells, f_hi=a.f_hi, seed=a.seed)
    srv = Server(meshes, a.precision, workers=a.workers, max_queue=a.max_queue or None)
    out = run_trace(srv, trace)
    srv.close()
    out.update({"precision": a.precision, "rate": a.rate, "duration_s": a.duration, "workers": a.workers,
                "mesh_setup_s": setup, "cells": cells, "max_queue": a.max_queue or None, "calibration": calib})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
