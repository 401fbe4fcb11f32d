"""The multi-GPU path's host logic with two processes on CPU (gloo): the
bench's replicas each time their own batch, the job lasts as long as the
slowest rank (max over ranks), the whole-job rate counts every rank's work,
and the reference arm runs on rank 0 only.  On GPUs the same functions run
under NCCL (bench.py under torchrun); the path has no data collective, only
these reductions and barriers."""
import json
import multiprocessing as mp
import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    bench.barrier(world)
    slowest = bench.max_over_ranks(1.0 + rank, world)
    rate, t = bench.weak_scaling_rate(1000.0, 0.5 * (rank + 1), world)
    bench.barrier(world)
    dist.destroy_process_group()
    Path(out, f"r{rank}.json").write_text(json.dumps({"slowest": slowest, "rate": rate, "t": t}))


def test_two_ranks_reduce_like_the_bench(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["slowest"] == 2.0          # max over ranks
        assert r["t"] == 1.0                # the slowest rank's time
        assert r["rate"] == 2000.0          # every rank's units over the slowest time


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun every rank starts bench.py --impl reference; ranks
    other than 0 return at once without work."""
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse_args()) == 0
