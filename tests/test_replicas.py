"""The multi-process path of ``bench.py``: N ranks are independent replicas of the one-GPU path,
joined only by a barrier around the timed region and the max of their times.  Here two ``gloo``
ranks on the CPU exercise that plumbing (``bench.Replicas``) and the reference arm's rule that
only rank 0 works and prints."""
import json
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    try:
        reps = bench.Replicas("gloo", timeout_s=60)
        reps.barrier()
        per_rank_ms = 10.0 * (rank + 1)            # rank 1 is the slower one
        ms = reps.max(per_rank_ms)
        q.put((rank, reps.world, ms, reps.rate(1000, ms / 1000.0)))
        reps.barrier()
        reps.close()
    except Exception as e:                          # reported to the parent, never hangs it
        q.put((rank, "error", repr(e), None))


def test_two_gloo_ranks_take_the_max_time_and_the_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    assert all(g[1] == 2 for g in got), got
    # both ranks see the slower rank's time, and the rate counts both replicas' cells
    assert [g[2] for g in got] == [20.0, 20.0]
    assert [g[3] for g in got] == [2 * 1000 / 0.020] * 2


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.delenv("RANK", raising=False)
    sys.path.insert(0, str(ROOT))
    import bench
    reps = bench.Replicas("gloo")
    assert reps.world == 1 and reps.rank == 0
    assert reps.max(3.5) == 3.5 and reps.rate(100, 0.5) == 200.0
    reps.barrier()
    reps.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    sys.path.insert(0, str(ROOT))
    import bench
    bench.main(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"])
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("n", [2000])
def test_reference_arm_line_on_rank_zero(monkeypatch, capsys, n):
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    sys.path.insert(0, str(ROOT))
    import bench
    bench.main(["--impl", "reference", "--steps", "1", "--warmup", "3", "--n", str(n),
                "--ref-budget", "1"])
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "cells/s" and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "cells/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
