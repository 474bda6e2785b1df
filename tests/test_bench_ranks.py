"""The multi-rank plumbing of bench.py on CPU (no GPU): two `gloo` ranks
time different step lengths and must both take the slower one (the job is
as slow as its slowest replica), the job throughput counts every replica's
cell-updates, and the reference arm runs on rank 0 alone."""
import json
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
        q.put((rank, ms, bench.job_throughput(world, 1_000_000, ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _, _ in out) == [0, 1]
    for _, ms, thr in out:
        assert ms == 15.0
        assert thr == pytest.approx(2 * 1_000_000 / 15e-3 * 1e-6)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.job_throughput(1, 2_000_000, 4.0) == pytest.approx(500.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    calls = []

    def fake_run(bs, steps, threads):
        calls.append((steps, threads))
        return {"mcell_updates_per_s": 12.5, "seconds": 0.4, "threads": 3}

    monkeypatch.setattr(bench, "cpu_reference_run", fake_run)
    args = bench.parse_args(["--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1"])
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(args) is None
    assert calls == [] and capsys.readouterr().out == ""
    monkeypatch.setenv("RANK", "0")
    bench.run_reference(args)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert len(calls) == 3
    assert line["impl"] == "reference" and line["value"] == 12.5 and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 3
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
