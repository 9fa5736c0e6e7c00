"""CPU: the multi-GPU mode's host plumbing with two ranks on gloo.

The inverter path runs as independent replicas, one process per GPU; the ranks
share only the timed-run plumbing of cl2qcd_b200.replicas (a barrier on both
sides of the timed region, the maximum of the per-rank times, the whole-job
rate).  Two processes (spawned, as torchrun would start them) run it over gloo
here; the bench's reference arm, started on every rank by torchrun, must do its
work on rank 0 only.
"""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    from cl2qcd_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=30)
    r.barrier()
    t_max = r.max_over_ranks(1.0 + rank)  # rank 1 is the slow one
    rate = r.rate(10.0, 1.0 + rank)       # 10 units per rank
    r.barrier()
    r.close()
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump({"world": r.world, "rank": r.rank, "t_max": t_max, "rate": rate}, f)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    for k, r in enumerate(res):
        assert (r["world"], r["rank"]) == (world, k)
        assert r["t_max"] == 2.0            # every rank sees the slowest rank's time
        assert r["rate"] == pytest.approx(world * 10.0 / 2.0)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    from cl2qcd_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.pg is None and r.world == 1
    assert r.max_over_ranks(3.5) == 3.5 and r.rate(7.0, 2.0) == 3.5
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse()) == 0
    assert capsys.readouterr().out == ""
