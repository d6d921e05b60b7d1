"""Frequency replicas, the multi-GPU plan: every rank solves its own sweep,
with no data exchange, and the job's time is the slowest rank's. The plumbing
bench.py uses (aphi_b200.replicas) runs here on CPU ranks over gloo, world
size 2: the launcher environment, distinct per-rank frequencies, barriers, the
single max-over-ranks reduction of the timed figures and the whole-job rate."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from aphi_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, outdir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        r, w, local = replicas.dist_env()
        omegas = replicas.rank_omegas(r, 16, 50.0, 1e6)
        replicas.barrier()
        # per-rank sweep, e2e and FP64 times (ms): the job's are the maxima
        mx = replicas.max_over_ranks([100.0 + 10.0 * r, 200.0 - 50.0 * r, 300.0])
        replicas.barrier()
        rate = replicas.job_rate(w, 16, mx[0])
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"env": [r, w, local], "omegas": omegas.tolist(), "max": mx, "rate": rate}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    out = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, o in enumerate(out):
        assert o["env"] == [r, world, r]
        assert o["max"] == [110.0, 200.0, 300.0]          # the slowest rank's figure, on every rank
        assert o["rate"] == pytest.approx(2 * 16 / 0.110)  # all ranks' solves over the slowest time
    a, b = np.array(out[0]["omegas"]), np.array(out[1]["omegas"])
    assert a.size == b.size == 16 and not np.intersect1d(a, b).size   # ranks solve different systems
    np.testing.assert_allclose(b / a, 1.001)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.dist_env() == (0, 1, 0)
    replicas.barrier()
    assert replicas.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert replicas.job_rate(1, 16, 4000.0) == pytest.approx(4.0)
