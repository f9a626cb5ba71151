"""bench.py's multi-rank logic on the CPU: two gloo ranks (one process each,
rendezvous on 127.0.0.1) take the max over ranks, number their replicas
globally and aggregate throughput over the whole job; the reference arm runs
on rank 0 only.  The GPU arms use the same helpers with NCCL."""
from __future__ import annotations

import argparse
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        w, r, _ = bench.dist_env()
        # per-rank step times: the job runs at the slowest rank's pace
        ms = bench.max_over_ranks(5.0 + 2.0 * r, w, device="cpu")
        seeds = [bench.replica_seed(11, r, 64, k) for k in range(64)]
        gathered = [None] * w
        dist.all_gather_object(gathered, seeds)
        out.put((r, w, ms, gathered, bench.aggregate_ns_per_day(w, 64, 2.0, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_timing_and_seeds():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for r, w, ms, gathered, value in results:
        assert w == 2
        assert ms == 7.0  # max over ranks of 5 and 7
        # 2 ranks x 64 replicas x 2 fs per 7 ms
        assert value == pytest.approx(2 * 64 * 2.0e-6 / 7.0e-3 * 86400.0)
        flat = [s for per_rank in gathered for s in per_rank]
        assert len(set(flat)) == 128  # every replica of the job seeded differently
    assert results[0][3] == results[1][3]


def test_single_rank_helpers():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_seed(0, 0, 64, 1) == 0xC0FFEE
    assert bench.replica_seed(0, 1, 64, 0) == 64 * 0xC0FFEE
    assert bench.aggregate_ns_per_day(1, 64, 2.0, 8.0) == pytest.approx(64 * 2e-6 / 8e-3 * 86400.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(gpus=2, steps=1, warmup=3, replicas=64, residues=300, dt=2.0, seed=0, cutoff=False,
                              no_sasa=False, sasa_gamma_scale=0.25)
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference(args) is None
    assert buf.getvalue() == ""
