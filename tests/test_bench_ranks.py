"""bench.py's multi-process host logic on the CPU: world-size-2 gloo ranks agree on the
max-over-ranks step time, the reference arm runs on rank 0 only, and a --gpus / WORLD_SIZE
mismatch is refused.  (Each GPU rank computes an independent product; the only collectives
are the barrier and this max.)"""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        step_ms = bench.ranks_reduce_max(dist, 10.0 + 3.0 * rank, "cpu")
        e2e_ms = bench.ranks_reduce_max(dist, 50.0 - rank, "cpu")
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"step_ms": step_ms, "e2e_ms": e2e_ms}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    assert all(g == {"step_ms": 13.0, "e2e_ms": 50.0} for g in got)


def test_single_process_needs_no_collective():
    assert bench.ranks_reduce_max(None, 7.5, "cpu") == 7.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                                      "--warmup", "0"])
    assert bench.main() == 0
    assert capsys.readouterr().out == ""


def test_gpus_must_match_world_size(monkeypatch, capsys):
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2"])
    assert bench.main() == 2
    assert "WORLD_SIZE" in capsys.readouterr().err


def test_ours_requires_three_warmup_steps(monkeypatch, capsys):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--warmup", "2"])
    assert bench.main() == 2
