"""The multi-rank path of bench.py on the CPU: two gloo ranks, the job time
as the maximum over ranks (each rank's timed region ends at a barrier) and
the whole-job rate of independent replicas (weak scaling).  The DEM step does
not shard: N GPUs run N replicas and no collective touches the data path."""
import importlib.util
import json
import os
import pathlib
import socket
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    b = _bench()
    got_ws, got_rank, got_local = b.dist_env()
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    ms = 10.0 * (rank + 1)   # rank 1 is the slower replica
    max_ms = b.max_over_ranks(torch, dist, ms, torch.device("cpu"), ws)
    rate = b.whole_job_rate(500000, 20, ws, max_ms)
    dist.barrier()
    dist.destroy_process_group()
    (pathlib.Path(out_dir) / f"r{rank}.json").write_text(
        json.dumps({"env": [got_ws, got_rank, got_local], "max_ms": max_ms, "rate": rate}))


def test_two_gloo_ranks_take_the_max_time(tmp_path):
    import torch.multiprocessing as mp
    ws, port = 2, _free_port()
    mp.start_processes(_rank, args=(ws, port, str(tmp_path)), nprocs=ws, join=True, start_method="spawn")
    for r in range(ws):
        d = json.loads((tmp_path / f"r{r}.json").read_text())
        assert d["env"] == [ws, r, r]
        assert d["max_ms"] == 20.0                       # the slower rank's time, on every rank
        assert d["rate"] == pytest.approx(500000 * 20 * ws / 0.020)


def test_single_rank_needs_no_process_group():
    import torch
    b = _bench()
    assert b.max_over_ranks(torch, None, 7.5, torch.device("cpu"), 1) == 7.5
    assert b.whole_job_rate(1000, 10, 1, 2.0) == pytest.approx(5e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    b = _bench()
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = b.argparse.Namespace(steps=1, warmup=3, precision="mixed", gpus=2, impl="reference")
    assert b.run_reference(args) is None
    assert capsys.readouterr().out == ""
