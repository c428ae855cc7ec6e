"""The replica plumbing of bench.py on two gloo ranks (CPU): rendezvous,
the barrier, the max-over-ranks timing, the whole-job aggregate, and the
reference arm printing from rank 0 only.  On the GPU box the same code runs
over NCCL with one process per GPU."""
from __future__ import annotations

import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _, pg = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(pg)
        # the slowest rank's time is the job's time
        ms = bench.max_over_ranks(pg, 100.0 + 25.0 * rank)
        bench.barrier(pg)
        out.put((r, w, ms, bench.job_mlups(w, 1000, 10, ms)))
    finally:
        pg.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_barrier_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    for _, w, ms, mlups in res:
        assert w == 2 and ms == 125.0
        # 2 replicas x 1000 cells x 10 steps in 125 ms
        assert mlups == pytest.approx(2 * 1000 * 10 / 0.125 / 1e6)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, gpus = 2, 3, 2

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    assert bench.reference_arm(Args()) == 0
    assert capsys.readouterr().out == ""
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("LBM_REF_BUDGET_S", "1")
    assert bench.reference_arm(Args()) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
