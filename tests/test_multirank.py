"""The N > 1 path on CPU: bench.py runs one replica per rank (every grid
independent, no data-path collective) and reports the slowest rank's time and
all ranks' bytes.  Two gloo ranks on 127.0.0.1 check that every rank gets the
same maximum, the whole-job throughput counts both replicas, and the
reference arm prints on rank 0 only."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
    got = bench.max_over_ranks(ms, world, "cpu")
    gbs = bench.whole_job_gbs(1e9, got, world)
    dist.barrier()
    dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"ms": got, "gbs": gbs}))


def test_two_gloo_ranks_agree_on_the_slowest_replica(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert res[0]["ms"] == res[1]["ms"] == 15.0
    # two replicas of 1 GB each in 15 ms
    assert res[0]["gbs"] == pytest.approx(2 * 1e9 / 15e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.whole_job_gbs(1e9, 10.0, 1) == pytest.approx(100.0)


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_line_carries_the_contract_keys():
    p = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference",
                        "--steps", "3", "--warmup", "3", "--grid-edge", "64"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    sys.path.insert(0, str(REPO))
    import bench

    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "GB/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["steps"] == 3 and line["warmup"] == 3 and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("reference", "port")
    assert cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "adi_256cube_fp64_general_50iter"


def test_gpus_n_without_torchrun_spawns_n_ranks():
    # `bench.py --gpus 2` outside torchrun launches two ranks itself
    # (torch.distributed.run on 127.0.0.1); the reference arm then runs on
    # rank 0 alone, which prints the one JSON line, and rank 1 exits cleanly
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    p = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3", "--grid-edge", "32"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["config"]["iters_per_step"] == 50 and line["value"] > 0
