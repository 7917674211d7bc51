"""Multi-rank logic of bench.py on CPU (gloo, world size 2).

The timed region ends with the barrier and the reductions of the whole job
(max of the device time over ranks, sum of the cells).  These tests run that
logic in two gloo processes, check that the reference arm runs on rank 0
alone, and that `--gpus N` starts its N ranks itself.  (The partition of the
pair queue and the gather of the results are tested in
test_shards_multirank.py.)
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_setup("gloo")
    assert (r, w) == (rank, world)
    # Each rank's reads come from its own seed (weak scaling).
    profiles, _ = bench.make_profiles(20261205, 3)
    steps = bench.make_steps(bench.rank_seed(20261205, r), profiles, 1, 4)
    cells = float(1000 * (r + 1))
    ms = 10.0 * (r + 1)
    bench.barrier(w)
    value, ms_max, cells_all = bench.aggregate(cells, ms, w)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"value": value, "ms_max": ms_max, "cells_all": cells_all, "first_read": steps[0][0]}, f)
    dist.destroy_process_group()


def test_ranks_shard_reads_and_reduce_time_and_cells(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["ms_max"] == 20.0  # the slowest rank's time
        assert r["cells_all"] == 3000.0  # every rank's cells
        assert r["value"] == pytest.approx(3000.0 / 0.020 / 1e9)
    assert res[0]["first_read"] != res[1]["first_read"]  # disjoint work per rank


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    args = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
            "--warmup", "0", "--reads-per-step", "4", "--profiles", "2", "--cpu-seconds", "0.5"]
    res = subprocess.run(args, env=env, capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.strip() == ""  # no line, no work, no process group
    env["RANK"] = env["LOCAL_RANK"] = "0"
    res = subprocess.run(args, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads([l for l in res.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1


def test_gpus_flag_launches_the_ranks_itself(tmp_path):
    """`bench.py --gpus 2` without a launcher starts two ranks (torchrun on
    127.0.0.1); the reference arm then prints one line, from rank 0, with
    n_gpus 2."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    args = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
            "--warmup", "0", "--reads-per-step", "4", "--profiles", "2", "--cpu-seconds", "0.5"]
    res = subprocess.run(args, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
